"""CPU tests of the C-ABI library's host side: exported symbols, octree,
interaction lists, operator tables and error behaviour.  No GPU needed: the
set-up phase (rtfmm_b200_setup) touches no device."""
import math
import os
import re

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "rtfmm_b200.h")


def header_symbols():
    src = open(HEADER).read()
    return sorted(set(re.findall(r"\b(rtfmm_b200_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.lib()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(pkg.rtfmm.EXPORTS)
    assert b"sm_100a" in L.rtfmm_b200_version()


def uniform(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 3)) - 0.5
    q = rng.random(n) * 2 - 1
    return x, q - q.mean()


def blobs(n, nblob, sigma, seed):
    rng = np.random.default_rng(seed)
    c = rng.random((nblob, 3))
    x = c[rng.integers(0, nblob, n)] + sigma * rng.standard_normal((n, 3))
    x = np.mod(x, 1.0) - 0.5
    q = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    return x, q - q.mean()


def lists_of(f):
    pi, po = f.p2p_lists()
    p2p = sorted((int(a), int(b), tuple(np.round(o, 12))) for (a, b), o in zip(pi, po))
    mi, mo = f.m2l_lists()
    m2l = sorted((int(a), int(b), int(c), tuple(np.round(o, 12))) for (a, b, c), o in zip(mi, mo))
    return p2p, m2l


def oracle_lists(F):
    p2p = sorted((t, s, tuple(np.round(off, 12))) for t, l in F.trav.p2p.items() for (s, off) in l)
    m2l = sorted((t, s, sg, tuple(np.round(off, 12))) for t, l in F.trav.m2l_parent.items()
                 for (s, off, sg) in l)
    return p2p, m2l


CASES = [
    ("uniform", 3000, 32, 0), ("uniform", 3000, 32, 1), ("uniform", 2500, 16, 3),
    ("blobs", 4000, 16, 2), ("single_leaf", 50, 64, 2), ("tiny", 9, 1, 1),
]


@pytest.mark.parametrize("kind,n,ncrit,images", CASES)
def test_tree_and_lists_match_oracle(pkg, oracle, kind, n, ncrit, images):
    if kind == "blobs":
        x, q = blobs(n, 4, 0.03, 7)
    else:
        x, q = uniform(n, n)
    f = pkg.LaplaceFMM(x, q, pkg.Argument(P=4, ncrit=ncrit, images=images, cycle=1.0))
    f.setup()
    F = oracle.FMM(x, q, 4, ncrit, images, 1.0)
    ints, reals = f.cells()
    C = F.cells
    assert len(C) == ints.shape[0]
    for c in range(len(C)):
        assert tuple(ints[c, :6]) == (C.octant[c], C.depth[c], C.coff[c], C.cnum[c], C.boff[c], C.bnum[c])
        assert reals[c, 0] == C.r[c]
        assert tuple(reals[c, 1:]) == tuple(C.x[c])
    assert np.array_equal(f.perm(), F.perm)
    assert lists_of(f) == oracle_lists(F)
    # each target's P2P list in the reference's recursion order (the order
    # of the FP64 sums), also when the walk is split across threads
    pi, po = f.p2p_lists()
    got = {}
    for (t, s_), o in zip(pi, po):
        got.setdefault(int(t), []).append((int(s_), tuple(np.round(o, 12))))
    want = {t: [(s_, tuple(np.round(off, 12))) for (s_, off) in l] for t, l in F.trav.p2p.items() if l}
    assert got == want


def test_m2l_parent_map_is_symmetric(pkg):
    """Every 8x8 parent pair appears in both directions with opposite offsets
    (the transposed chain of the adjoint relies on it)."""
    x, q = uniform(4000, 11)
    f = pkg.LaplaceFMM(x, q, pkg.Argument(P=4, ncrit=24, images=2, cycle=1.0))
    f.setup()
    mi, mo = f.m2l_lists()
    s = {(int(a), int(b), tuple(np.round(o, 12))) for (a, b, c), o in zip(mi, mo) if c == 0}
    for (a, b, o) in s:
        assert (b, a, tuple(-v + 0.0 for v in o)) in s


def test_p2p_lists_symmetric(pkg):
    x, q = blobs(3000, 3, 0.05, 5)
    f = pkg.LaplaceFMM(x, q, pkg.Argument(P=4, ncrit=20, images=1, cycle=1.0))
    f.setup()
    pi, po = f.p2p_lists()
    s = {(int(a), int(b), tuple(np.round(o, 12))) for (a, b), o in zip(pi, po)}
    for (a, b, o) in s:
        assert (b, a, tuple(-v + 0.0 for v in o)) in s


@pytest.mark.parametrize("P", [4, 6])
def test_kernel_spectra_match_oracle(pkg, oracle, P):
    """8x8 sibling spectra (precompute_m2l, kernel.cpp:1783-1811): the
    library's host DFT against numpy's rfftn in the oracle."""
    x, q = uniform(200, 1)
    f = pkg.LaplaceFMM(x, q, pkg.Argument(P=P, ncrit=64, images=2, cycle=1.0))
    f.setup()
    N = 2 * P - 1
    Nf = N * N * P
    got = f.operator(3, 26 * 64 * Nf * 2).reshape(26, 8, 8, Nf, 2)
    got = got[..., 0] + 1j * got[..., 1]
    ops = oracle.Operators(P, 0.5, 2)
    ref = ops.cc8.reshape(26, 8, 8, Nf)
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() / scale < 1e-13


@pytest.mark.parametrize("P", [4, 6, 8, 10])
def test_m2m_reproduces_child_potential(pkg, oracle, P):
    """The parent equivalent density from M2M reproduces the child's field on
    the parent check surface (the defining property of the operator,
    kernel.cpp:1660-1668), and the library's pseudo-inverse agrees with the
    oracle's in that sense."""
    x, q = uniform(200, 2)
    f = pkg.LaplaceFMM(x, q, pkg.Argument(P=P, ncrit=64, images=1, cycle=1.0))
    f.setup()
    ns = oracle.surface_point_num(P)
    m2m = f.operator(1, 8 * ns * ns).reshape(8, ns, ns)
    r0 = 0.5
    xc = oracle.surface_points(P, r0 * 2.95)
    xe = oracle.surface_points(P, r0 * 1.05)
    A = oracle.p2p_matrix(xe, xc)
    rng = np.random.default_rng(P)
    for o in range(8):
        xch = oracle.surface_points(P, r0 / 2 * 1.05, oracle.child_center(np.zeros(3), r0, o))
        G = oracle.p2p_matrix(xch, xc)
        qc = rng.standard_normal(ns)
        target = G @ qc
        err = np.linalg.norm(A @ (m2m[o] @ qc) - target) / np.linalg.norm(target)
        assert err < {4: 1e-12, 6: 1e-10, 8: 1e-8, 10: 1e-9}[P]


@pytest.mark.parametrize("P", [8, 10])
def test_svd_factors_are_orthonormal(pkg, oracle, P):
    """U and V of the check-to-equivalent operator are orthonormal to working
    precision, as an orthogonal factorisation (the reference's dgesvd,
    mathfunc.cpp:81-110) returns them, also at P = 10 where the operator's
    condition number (1.3e16) exceeds 1/eps: U = A V / s alone loses
    orthogonality in the columns of the smallest singular values."""
    x, q = uniform(200, 3)
    f = pkg.LaplaceFMM(x, q, pkg.Argument(P=P, ncrit=64, images=1, cycle=1.0))
    f.setup()
    ns = oracle.surface_point_num(P)
    U = f.operator(4, ns * ns).reshape(ns, ns)
    VS = f.operator(5, ns * ns).reshape(ns, ns)
    sinv = np.linalg.norm(VS, axis=0)
    keep = sinv > 0
    V = VS[:, keep] / sinv[keep]
    assert np.abs(U.T @ U - np.eye(ns)).max() < 1e-13
    assert np.abs(V.T @ V - np.eye(int(keep.sum()))).max() < 1e-13


def test_errors(pkg):
    x, q = uniform(100, 3)
    with pytest.raises(pkg.RtfmmError) as e:
        pkg.LaplaceFMM(x, q, pkg.Argument(P=1))
    assert e.value.code == 1
    with pytest.raises(pkg.RtfmmError):
        pkg.LaplaceFMM(x, q[:-1], pkg.Argument(P=4))
    bad = x.copy()
    bad[3, 1] = np.nan
    f = pkg.LaplaceFMM(bad, q, pkg.Argument(P=4))
    with pytest.raises(pkg.RtfmmError) as e:
        f.setup()
    assert e.value.code == 1
    # more than ncrit coincident bodies: the reference would split forever
    same = np.zeros((40, 3))
    f = pkg.LaplaceFMM(same, np.ones(40), pkg.Argument(P=4, ncrit=8))
    with pytest.raises(pkg.RtfmmError) as e:
        f.setup()
    assert "deeper" in str(e.value)
    # out of order
    f = pkg.LaplaceFMM(x, q, pkg.Argument(P=4))
    with pytest.raises(pkg.RtfmmError) as e:
        f.download()
    assert e.value.code == 4


def test_empty_input_setup(pkg):
    f = pkg.LaplaceFMM(np.zeros((0, 3)), np.zeros(0), pkg.Argument(P=4, images=2, cycle=1.0))
    f.setup()
    assert f.info()["nleaf"] == 1


def test_generate_random_bodies_matches_oracle(pkg, oracle):
    x1, q1 = pkg.generate_random_bodies(500, math.pi, seed=5, zero_netcharge=1)
    x2, q2 = oracle.generate_random_bodies(500, math.pi, seed=5, zero_netcharge=1)
    assert np.array_equal(x1, x2) and np.array_equal(q1, q2)


def test_p2p_pairs_cover_reference_lists(pkg, oracle):
    """The reference's P2P lists may pair a non-leaf cell with a leaf (its
    M2P/P2L-to-P2P conversions, traverser.cpp:75-86); the library expands
    those into leaf pairs.  The body-pair count must be unchanged."""
    x, q = blobs(5000, 5, 0.02, 3)
    f = pkg.LaplaceFMM(x, q, pkg.Argument(P=4, ncrit=32, images=3, cycle=1.0))
    f.setup()
    F = oracle.FMM(x, q, 4, 32, 3, 1.0)
    C = F.cells
    nonleaf = sum(1 for t, l in F.trav.p2p.items() for (s, off) in l if C.cnum[t] or C.cnum[s])
    assert nonleaf > 0
    pairs = sum(C.bnum[t] * C.bnum[s] for t, l in F.trav.p2p.items() for (s, off) in l)
    assert f.info()["p2p_pairs"] == pairs


@pytest.mark.parametrize("P", [4, 6])
def test_svd_factors(pkg, oracle, P):
    """The exported SVD factors: U is orthogonal and V S^-1 U^T is the
    pseudo-inverse of the equivalent-to-check matrix (kernel.cpp:1643-1651)."""
    x, q = uniform(200, 4)
    f = pkg.LaplaceFMM(x, q, pkg.Argument(P=P, ncrit=64, images=0, cycle=1.0))
    f.setup()
    ns = oracle.surface_point_num(P)
    U = f.operator(4, ns * ns).reshape(ns, ns)
    VS = f.operator(5, ns * ns).reshape(ns, ns)
    assert np.abs(U.T @ U - np.eye(ns)).max() < 1e-12
    xc = oracle.surface_points(P, 0.5 * 2.95)
    xe = oracle.surface_points(P, 0.5 * 1.05)
    A = oracle.p2p_matrix(xe, xc)
    pinv = VS @ U.T
    assert np.linalg.norm(A @ pinv @ A - A) / np.linalg.norm(A) < 1e-9
    assert np.allclose(pinv, f.operator(0, ns * ns).reshape(ns, ns), rtol=0, atol=1e-9 * np.abs(pinv).max())


def test_operator_tables_shared_between_handles(pkg):
    """A second handle with the same (P, images, cycle) copies the cached
    operator tables (bit for bit) instead of building them; clearing the
    cache makes the next set-up build them again."""
    x, q = uniform(300, 4)
    a = pkg.Argument(P=6, ncrit=32, images=2, cycle=1.0)
    pkg.clear_operator_cache()
    f1 = pkg.LaplaceFMM(x, q, a)
    f1.setup()
    t1 = f1.setup_times()["operators"]
    f2 = pkg.LaplaceFMM(x, q, a)
    f2.setup()
    t2 = f2.setup_times()["operators"]
    ns = 152
    for which, size in [(0, ns * ns), (1, 8 * ns * ns), (2, ns * ns), (4, ns * ns), (5, ns * ns), (7, ns * ns)]:
        assert np.array_equal(f1.operator(which, size), f2.operator(which, size))
    assert t2 < t1 / 3, (t1, t2)
    # the build's parts add up to the operator phase; a cached set reports none
    st1, st2 = f1.setup_times(), f2.setup_times()
    parts = ("ops_svd", "ops_orth", "ops_m2m", "ops_img", "ops_spectra", "ops_blocks")
    assert all(st1[k] >= 0 for k in parts) and st1["ops_svd"] > 0
    assert 0.5 * t1 <= sum(st1[k] for k in parts) <= t1 * 1.01 + 1e-4, st1
    assert all(st2[k] == 0 for k in parts), st2
    pkg.clear_operator_cache()
    f3 = pkg.LaplaceFMM(x, q, a)
    f3.setup()
    assert np.array_equal(f1.operator(1, 8 * ns * ns), f3.operator(1, 8 * ns * ns))
    for f in (f1, f2, f3):
        f.close()


def test_operator_tables_saved_and_loaded(pkg, tmp_path):
    """Tables written by save_operators and loaded in a (simulated) later
    process equal the built ones bit for bit and spare the build; files that
    do not match are refused."""
    x, q = uniform(300, 5)
    a = pkg.Argument(P=5, ncrit=32, images=2, cycle=1.0)
    pkg.clear_operator_cache()
    f1 = pkg.LaplaceFMM(x, q, a)
    f1.setup()
    t_build = f1.setup_times()["operators"]
    path = str(tmp_path / "ops_p5.bin")
    f1.save_operators(path)
    pkg.clear_operator_cache()
    pkg.load_operators(path)
    f2 = pkg.LaplaceFMM(x, q, a)
    f2.setup()
    assert f2.setup_times()["operators"] < t_build / 3
    ns = 6 * 4 ** 2 + 2
    N = 9
    nf = N * N * (N // 2 + 1)
    for which, size in [(0, ns * ns), (1, 8 * ns * ns), (2, ns * ns), (3, 26 * 64 * nf * 2), (4, ns * ns),
                        (5, ns * ns)]:
        assert np.array_equal(f1.operator(which, size), f2.operator(which, size)), which
    # malformed files
    raw = open(path, "rb").read()
    bad = tmp_path / "bad.bin"
    for blob in (raw[: len(raw) // 2], b"NOTOPS!!" + raw[8:], raw + b"x"):
        bad.write_bytes(blob)
        with pytest.raises(pkg.RtfmmError) as e:
            pkg.load_operators(str(bad))
        assert e.value.code == 1
    with pytest.raises(pkg.RtfmmError):
        pkg.load_operators(str(tmp_path / "missing.bin"))
    pkg.clear_operator_cache()
    for f in (f1, f2):
        f.close()


@pytest.mark.parametrize("kind,n,ncrit,images,precision", [
    ("uniform", 3000, 32, 2, 0), ("blobs", 4000, 8, 1, 1), ("blobs", 2500, 4, 0, 0)])
def test_leaf_lists_expand_the_reference_lists(pkg, kind, n, ncrit, images, precision):
    """The pass's leaf-to-leaf P2P lists are the reference's cell lists with
    every pair of a leaf and a non-leaf cell expanded into the leaves beneath
    it: for each target leaf, the lists of its ancestors from the root down
    (and its own), entries in list order, each source's leaves in
    first-body order."""
    x, q = (uniform(n, 21) if kind == "uniform" else blobs(n, 3, 0.01, 22))
    f = pkg.LaplaceFMM(x, q, pkg.Argument(P=4, ncrit=ncrit, images=images, cycle=1.0, precision=precision))
    f.setup()
    ints, reals = f.cells()
    cnum, coff, boff, bnum = ints[:, 3], ints[:, 2], ints[:, 4], ints[:, 5]
    ntree = int(np.sum(ints[:, 1] >= 0))
    leaves = [c for c in range(ntree) if cnum[c] == 0]
    leaf_index = {c: i for i, c in enumerate(leaves)}
    parent = {}
    for c in range(ntree):
        for k in range(cnum[c]):
            parent[coff[c] + k] = c
    by_first_body = sorted(leaves, key=lambda c: boff[c])
    pi, po = f.p2p_lists()
    lists = {}
    for (t, s_), o in zip(pi, po):
        lists.setdefault(int(t), []).append((int(s_), o))

    first = np.array([boff[l] for l in by_first_body])

    def leaves_under(c):
        a, b = np.searchsorted(first, [boff[c], boff[c] + bnum[c]])
        return by_first_body[a:b]

    lo, src, off = f.leaf_lists()
    assert len(lo) == len(leaves) + 1
    for i, c in enumerate(leaves):
        path = [c]
        while path[-1] in parent:
            path.append(parent[path[-1]])
        want = []
        for a in reversed(path):
            for s_, o in lists.get(a, []):
                want += [(leaf_index[l], o) for l in leaves_under(s_)]
        got_src = src[lo[i]:lo[i + 1]].tolist()
        assert got_src == [w[0] for w in want], c
        assert np.allclose(off[lo[i]:lo[i + 1]], np.array([w[1] for w in want]).reshape(-1, 3), atol=1e-12), c
    f.close()


def test_create_rejects_unknown_dipole_mode(pkg):
    import ctypes
    L = pkg.lib()
    a = pkg.rtfmm._Args()
    L.rtfmm_b200_default_args(ctypes.byref(a))
    h = ctypes.c_void_p()
    for mode, ok in ((0, True), (1, True), (2, True), (3, False), (-1, False)):
        a.dipole_correction = mode
        rc = L.rtfmm_b200_create(ctypes.byref(a), ctypes.byref(h))
        assert (rc == 0) == ok, mode
        if rc == 0:
            L.rtfmm_b200_destroy(h)
