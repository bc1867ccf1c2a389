"""The construction of the GPU octree, checked on the CPU.

The device builder (exafmm-rd_b200/csrc/rtfmm_tree.cu) computes each body's
octant digits for levels 1..21 with the host split's comparisons and centre
arithmetic, sorts (key, index) stably, splits each level's cells that hold
more than ncrit bodies by binary search on the next digit (children in
(parent, octant) order), and puts each leaf's bodies back in input order.
This test runs that construction in numpy and requires the oracle's
Tree::build_nonuniform_octree (3dpp/src/tree.cpp:102-188) cells and body
permutation exactly, including bodies that sit exactly on cell centres.
"""
import numpy as np
import pytest

LEVELS = 21


def path_keys(x, center, r0):
    n = len(x)
    c = np.tile(np.asarray(center, dtype=np.float64), (n, 1))
    r = np.full(n, r0)
    key = np.zeros(n, dtype=np.uint64)
    for _ in range(LEVELS):
        o = ((x[:, 0] > c[:, 0]).astype(np.uint64) << np.uint64(2)) | \
            ((x[:, 1] > c[:, 1]).astype(np.uint64) << np.uint64(1)) | (x[:, 2] > c[:, 2]).astype(np.uint64)
        key = (key << np.uint64(3)) | o
        h = r / 2
        for k, bit in ((0, 4), (1, 2), (2, 1)):
            c[:, k] = c[:, k] + np.where((o & np.uint64(bit)) != 0, h, -h)
        r = h
    return key


def build_by_keys(x, center, r0, ncrit):
    n = len(x)
    key = path_keys(x, center, r0)
    order = np.argsort(key, kind="stable")
    skey = key[order]
    # cells: octant, depth, r, centre, coff, cnum, boff, bnum (breadth first)
    cells = [[13, 0, r0, np.asarray(center, dtype=np.float64), 0, 0, 0, n]]
    lev0, lev1 = 0, 1
    while lev0 < lev1:
        for ci in range(lev0, lev1):
            octant, depth, r, cx, _, _, b0, nb = cells[ci]
            if nb <= ncrit:
                continue
            assert depth < LEVELS
            shift = np.uint64(3 * (LEVELS - 1 - depth))
            digit = ((skey[b0:b0 + nb] >> shift) & np.uint64(7)).astype(np.int64)
            start = np.searchsorted(digit, np.arange(9), side="left")
            start[8] = nb
            first = len(cells)
            k = 0
            for o in range(8):
                cnt = int(start[o + 1] - start[o])
                if cnt == 0:
                    continue
                s = np.array([1.0 if o & 4 else -1.0, 1.0 if o & 2 else -1.0, 1.0 if o & 1 else -1.0])
                cells.append([o, depth + 1, r / 2, cx + s * (r / 2), 0, 0, b0 + int(start[o]), cnt])
                k += 1
            cells[ci][4], cells[ci][5] = first, k
        lev0, lev1 = lev1, len(cells)
    # input order inside each leaf
    perm = order.copy()
    for octant, depth, r, cx, coff, cnum, b0, nb in cells:
        if cnum == 0:
            perm[b0:b0 + nb] = np.sort(perm[b0:b0 + nb])
    return cells, perm


def lattice(m):
    g = (np.arange(m) + 0.5) / m
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)


@pytest.mark.parametrize("name,ncrit", [("uniform", 8), ("blobs", 4), ("lattice", 20)])
def test_key_construction_equals_the_host_split(oracle, name, ncrit):
    rng = np.random.default_rng(11)
    if name == "uniform":
        x = rng.random((3000, 3))
    elif name == "blobs":
        c = rng.random((4, 3))
        x = np.mod(c[rng.integers(0, 4, 3000)] + 0.003 * rng.standard_normal((3000, 3)), 1.0)
    else:
        x = lattice(16)  # sites at (i + 1/2)/16: some fall exactly on cell centres
    center = (0.5, 0.5, 0.5)
    cells, perm = build_by_keys(x, center, 0.5, ncrit)
    want, wperm = oracle.build_nonuniform_octree(x, np.asarray(center), 0.5, ncrit)
    assert np.array_equal(perm, wperm)
    assert len(cells) == len(want)
    for i, (octant, depth, r, cx, coff, cnum, b0, nb) in enumerate(cells):
        assert (octant, depth, coff, cnum, b0, nb) == (want.octant[i], want.depth[i], want.coff[i], want.cnum[i],
                                                      want.boff[i], want.bnum[i]), i
        assert r == want.r[i] and np.array_equal(cx, want.x[i]), i
