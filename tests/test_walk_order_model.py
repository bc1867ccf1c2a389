"""The ordering argument of the GPU P2P walk, checked on the CPU.

The GPU walk (exafmm-rd_b200/csrc/rtfmm_lists.cu) expands the dual-tree walk
breadth first, one frontier per level of the frame tree, gives every frame
its path (walk index, then the child index taken at each division) packed
into fixed-width keys, and recovers the recursion's list order by sorting
the emitted pairs by path and then, stably, by target.  This test runs that
construction in Python on the oracle's cells, with the frame step of
Traverser::horizontal_origin (3dpp/src/traverser.cpp:70-148) restated, and
requires the oracle's depth-first lists (order included).
"""
import numpy as np
import pytest

DIGITS = 40  # 19 in the first key word, 21 in the second


def uniform01(n, seed):
    rng = np.random.default_rng(seed)
    return rng.random((n, 3)), rng.random(n) * 2 - 1


def blobs(n, nblob, sigma, seed):
    rng = np.random.default_rng(seed)
    c = rng.random((nblob, 3))
    x = np.mod(c[rng.integers(0, nblob, n)] + sigma * rng.standard_normal((n, 3)), 1.0)
    return x, np.ones(n)


def step(c, adjacent, frame, off):
    """One frame: ("hit", source) | ("divide", [child frames]) | ("none",)."""
    tc, sc, tcp, scp = frame
    leaf = lambda k: c.cnum[k] == 0
    divide = 0
    if not adjacent(tc, sc, off):
        if adjacent(tc, scp, off) and leaf(tc) and c.depth[scp] >= c.depth[tc]:
            return ("hit", sc)
        if adjacent(tcp, sc, off) and leaf(sc) and c.depth[tcp] >= c.depth[sc]:
            return ("hit", sc)
        if adjacent(tcp, scp, off) and c.depth[tcp] == c.depth[scp]:
            return ("none",)
        if leaf(tc) and leaf(sc):
            return ("none",)
        divide = 1 if (not leaf(tc) and leaf(sc)) else 2 if (leaf(tc) and not leaf(sc)) else (
            1 if c.r[tc] >= c.r[sc] else 2)
    else:
        if leaf(tc) and leaf(sc):
            return ("hit", sc)
        divide = 1 if (not leaf(tc) and leaf(sc)) else 2 if (leaf(tc) and not leaf(sc)) else (
            1 if c.r[tc] >= c.r[sc] else 2)
    if divide == 1:
        return ("divide", [(c.coff[tc] + i, sc, tc, scp) for i in range(c.cnum[tc])])
    return ("divide", [(tc, c.coff[sc] + i, tcp, sc) for i in range(c.cnum[sc])])


def breadth_first_lists(T, roots):
    """roots: [(frame, offset)] in walk order.  Returns {target: [(src, off)]}."""
    c = T.cells
    frontier = [(fr, w, ()) for w, (fr, _) in enumerate(roots)]
    hits = []
    while frontier:
        nxt = []
        for fr, w, path in frontier:
            r = step(c, T.adjacent, fr, roots[w][1])
            if r[0] == "hit":
                hits.append((fr[0], r[1], w, path))
            elif r[0] == "divide":
                assert len(path) < DIGITS
                for i, kid in enumerate(r[1]):
                    nxt.append((kid, w, path + (i,)))
        frontier = nxt
    # fixed-width keys: the walk index, then the digits, zero-padded
    key = lambda h: (h[2],) + h[3] + (0,) * (DIGITS - len(h[3]))
    hits.sort(key=key)                      # depth-first order
    hits.sort(key=lambda h: h[0])           # stably by target
    out = {}
    for tc, sc, w, _ in hits:
        out.setdefault(tc, []).append((sc, roots[w][1]))
    return out


@pytest.mark.parametrize("make,ncrit,images", [
    (lambda: uniform01(600, 1), 16, 0),
    (lambda: uniform01(800, 2), 8, 1),
    (lambda: blobs(700, 3, 0.01, 3), 4, 2),
])
def test_breadth_first_path_keys_give_the_recursion_order(oracle, make, ncrit, images):
    x, q = make()
    F = oracle.FMM(x, q, 3, ncrit, images, 1.0, center=(0.5, 0.5, 0.5))
    T = F.trav
    c = T.cells
    if images == 0:
        roots = [((0, 0, 0, 0), np.zeros(3))]
    else:
        cidx = [k for k in range(len(c)) if c.depth[k] == -1][0]
        roots = [((0, 0, cidx, cidx), np.array([px, py, pz], dtype=np.float64))
                 for pz in (-1, 0, 1) for py in (-1, 0, 1) for px in (-1, 0, 1)]
    got = breadth_first_lists(T, roots)
    want = {t: l for t, l in T.p2p.items() if l}
    assert sorted(got) == sorted(want)
    for t in want:
        assert [s for s, _ in got[t]] == [s for s, _ in want[t]], t
        assert all(np.array_equal(a, b) for (_, a), (_, b) in zip(got[t], want[t])), t
