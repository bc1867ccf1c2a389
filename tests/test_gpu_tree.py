"""The octree built on the GPU from device-resident bodies
(rtfmm_b200_setup_device) against the host builder (rtfmm_b200_setup), which
the host-plan tests pin to the oracle's Tree::build_nonuniform_octree.

The two must give the same cells (octant, depth, children, body ranges,
centres and radii, bit for bit), the same body permutation, hence the same
lists, and the same pass outputs.  Cases: uniform bodies, clustered bodies
with a deep adaptive tree, a lattice whose sites fall exactly on cell
centres (the split compares with a strict >), leaves larger than a block,
a tree deeper than the 21 levels of the device keys (built on the host),
walks deep enough to need both words of the path keys, the C3 workload at
full size, no bodies at all, and non-finite input.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def uniform01(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 3))
    q = rng.random(n) * 2 - 1
    return x, q - q.mean()


def blobs(n, nblob, sigma, seed):
    rng = np.random.default_rng(seed)
    c = rng.random((nblob, 3))
    x = np.mod(c[rng.integers(0, nblob, n)] + sigma * rng.standard_normal((n, 3)), 1.0)
    q = np.where(rng.random(n) < 0.5, -1.0, 1.0)
    return x, q - q.mean()


def lattice(m):
    g = (np.arange(m) + 0.5) / m
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    q = np.where(np.arange(len(x)) % 2 == 0, 1.0, -1.0)
    return x, q


def deep_pair(seed):
    # two tight clusters 1e-9 wide: ncrit=4 needs ~33 levels
    rng = np.random.default_rng(seed)
    a = 0.3 + 1e-9 * rng.random((24, 3))
    b = 0.7 + 1e-9 * rng.random((24, 3))
    x = np.concatenate([a, b, rng.random((200, 3))])
    q = rng.standard_normal(len(x))
    return x, q - q.mean()


def build_both(pkg, x, q, **kw):
    a = pkg.Argument(cycle=1.0, x=(0.5, 0.5, 0.5), dipole_correction=0, divide_4pi=1, **kw)
    h = pkg.LaplaceFMM(x, q, a)
    h.setup()
    d = pkg.LaplaceFMM(x, q, a)
    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    qd = torch.from_numpy(np.ascontiguousarray(q)).cuda()
    d.setup_device(xd.data_ptr(), qd.data_ptr(), len(q))
    return h, d


CASES = [
    ("uniform", lambda: uniform01(30000, 41), dict(P=4, ncrit=32, images=2, precision=0)),
    ("blobs", lambda: blobs(40000, 6, 0.005, 42), dict(P=5, ncrit=16, images=1, precision=1)),
    ("lattice", lambda: lattice(24), dict(P=4, ncrit=20, images=3, precision=0)),
    ("big_leaves", lambda: uniform01(20000, 43), dict(P=4, ncrit=1000, images=0, precision=1)),
    ("deeper_than_keys", lambda: deep_pair(44), dict(P=4, ncrit=4, images=2, precision=0)),
    # tight clusters and tiny leaves: walks of more than 19 divisions (the
    # second word of the path keys)
    ("deep_walk", lambda: blobs(60000, 3, 0.0005, 47), dict(P=4, ncrit=4, images=1, precision=1)),
]


@pytest.mark.parametrize("name,make,kw", CASES, ids=[c[0] for c in CASES])
def test_device_tree_equals_host_tree(pkg, name, make, kw):
    x, q = make()
    h, d = build_both(pkg, x, q, **kw)
    # the pass: the device set-up leaves the bodies resident
    h.upload()
    h.evaluate_device()
    d.evaluate_device()
    ph, gh = h.download()
    pd, gd = d.download()
    assert np.array_equal(ph, pd) and np.array_equal(gh, gd)
    # the host-buffer calls on the device-built plan (they fetch the
    # set-up bodies from the device first): new charges, the adjoint
    q2 = np.random.default_rng(45).standard_normal(len(q))
    p2h, g2h = h.evaluate(q2)
    p2d, g2d = d.evaluate(q2)
    assert np.array_equal(p2h, p2d) and np.array_equal(g2h, g2d)
    w = np.random.default_rng(46).standard_normal(len(q))
    dqh, dxh = h.adjoint(w)
    dqd, dxd = d.adjoint(w)
    assert np.array_equal(dqh, dqd) and np.array_equal(dxh, dxd)
    # the plan itself
    hi, hr = h.cells()
    di, dr = d.cells()
    assert np.array_equal(hi, di) and np.array_equal(hr, dr)
    assert np.array_equal(h.perm(), d.perm())
    hp, ho = h.p2p_lists()
    dp, do = d.p2p_lists()
    assert np.array_equal(hp, dp) and np.array_equal(ho, do)
    hm = h.m2l_lists()
    dm = d.m2l_lists()
    assert all(np.array_equal(u, v) for u, v in zip(hm, dm))
    assert h.info() == d.info()
    # the pass's leaf lists, built on the host and on the GPU
    assert all(np.array_equal(u, v) for u, v in zip(h.leaf_lists(), d.leaf_lists()))
    st = d.setup_times()
    assert st["tree"] > 0 and st["total"] >= st["tree"]
    h.close()
    d.close()


def test_device_tree_empty_and_bad_input(pkg):
    a = pkg.Argument(P=4, ncrit=8, images=2, cycle=1.0, x=(0.5, 0.5, 0.5))
    f = pkg.LaplaceFMM(np.zeros((0, 3)), np.zeros(0), a)
    f.setup_device(0, 0, 0)
    assert f.info()["nleaf"] == 1
    assert f.evaluate_device() == 0
    f.close()
    x, q = uniform01(1000, 46)
    for bad_x in (True, False):
        xb, qb = x.copy(), q.copy()
        if bad_x:
            xb[17, 2] = np.inf
        else:
            qb[5] = np.nan
        f = pkg.LaplaceFMM(x, q, a)
        xd, qd = torch.from_numpy(xb).cuda(), torch.from_numpy(qb).cuda()
        with pytest.raises(pkg.RtfmmError) as e:
            f.setup_device(xd.data_ptr(), qd.data_ptr(), 1000)
        assert e.value.code == 1
        f.close()
    # more than ncrit coincident bodies: the same error as the host builder
    f = pkg.LaplaceFMM(np.zeros((40, 3)), np.ones(40), pkg.Argument(P=4, ncrit=8))
    xs = torch.zeros((40, 3), dtype=torch.float64, device="cuda")
    qs = torch.ones(40, dtype=torch.float64, device="cuda")
    with pytest.raises(pkg.RtfmmError) as e:
        f.setup_device(xs.data_ptr(), qs.data_ptr(), 40)
    assert "deeper" in str(e.value)
    f.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_resetup_reuses_buffers(pkg, precision):
    """One handle set up again and again (device and host set-up in turn, body
    sets growing and shrinking: its device buffers are reused or grown)
    gives the outputs of a fresh handle every time."""
    a = pkg.Argument(P=5, ncrit=32, images=2, cycle=1.0, x=(0.5, 0.5, 0.5), dipole_correction=0, divide_4pi=1,
                     precision=precision)
    x0, q0 = uniform01(100, 50)
    f = pkg.LaplaceFMM(x0, q0, a)
    for step, (n, dev) in enumerate([(20000, True), (5000, False), (40000, True), (12000, True), (30000, False)]):
        x, q = blobs(n, 3, 0.05, 60 + step) if step % 2 else uniform01(n, 60 + step)
        if dev:
            xd = torch.from_numpy(x).cuda()
            qd = torch.from_numpy(q).cuda()
            f.setup_device(xd.data_ptr(), qd.data_ptr(), n)
            f.evaluate_device()
            phi, grad = f.download()
        else:
            f.x, f.q, f.n = x, q, n
            phi, grad = f.solve()
        g = pkg.LaplaceFMM(x, q, a)
        rphi, rgrad = g.solve()
        g.close()
        assert np.array_equal(phi, rphi) and np.array_equal(grad, rgrad), step
    f.close()


@pytest.mark.parametrize("P,images", [(4, 2), (6, 0), (8, 3), (10, 3), (12, 1)])
def test_gpu_operators_equal_host(pkg, P, images):
    """A device set-up builds its operators on the GPU (the SVD sweeps, the
    M2M and image products and the kernel spectra); the tables equal the host
    set-up's bit for bit."""
    x, q = uniform01(500, 70 + P)
    a = pkg.Argument(P=P, ncrit=32, images=images, cycle=1.0, x=(0.5, 0.5, 0.5), dipole_correction=0)
    pkg.clear_operator_cache()  # each handle builds its own tables
    h = pkg.LaplaceFMM(x, q, a)
    h.setup()
    pkg.clear_operator_cache()
    d = pkg.LaplaceFMM(x, q, a)
    xd = torch.from_numpy(x).cuda()
    qd = torch.from_numpy(q).cuda()
    d.setup_device(xd.data_ptr(), qd.data_ptr(), len(q))
    assert d.setup_times()["operators"] > 0
    ns = 6 * (P - 1) ** 2 + 2
    N = 2 * P - 1
    nf = N * N * (N // 2 + 1)
    for which, size in [(0, ns * ns), (1, 8 * ns * ns), (2, ns * ns), (3, 26 * 64 * nf * 2), (4, ns * ns),
                        (5, ns * ns), (6, 26 * nf * 2), (7, ns * ns)]:
        assert np.array_equal(h.operator(which, size), d.operator(which, size)), which
    h.close()
    d.close()


def test_device_setup_at_c3_size(pkg):
    """The 2^22-body blob workload (P=10, ncrit=128, images=3): the device
    set-up's tree, permutation, lists and list sizes equal the host's."""
    x, q = blobs(1 << 22, 64, 0.02, 3)
    h, d = build_both(pkg, x, q, P=10, ncrit=128, images=3, precision=1)
    hi, hr = h.cells()
    di, dr = d.cells()
    assert np.array_equal(hi, di) and np.array_equal(hr, dr)
    assert np.array_equal(h.perm(), d.perm())
    hp, ho = h.p2p_lists()
    dp, do = d.p2p_lists()
    assert np.array_equal(hp, dp) and np.array_equal(ho, do)
    assert h.info() == d.info()
    h.close()
    d.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_solve_sets_up_on_the_gpu(pkg, precision):
    """rtfmm_b200_solve (the drop-in for LaplaceFMM::solve) builds the tree,
    lists and P2P tables on the GPU from 65536 bodies; its outputs equal the
    host set-up's bit for bit, and the set-up's phases show the device build
    (tree phase well under the host build's)."""
    x, q = blobs(1 << 17, 4, 0.05, 80)
    a = pkg.Argument(P=6, ncrit=64, images=3, cycle=1.0, x=(0.5, 0.5, 0.5), dipole_correction=0, divide_4pi=1,
                     precision=precision)
    f = pkg.LaplaceFMM(x, q, a)
    phi, grad = f.solve()
    g = pkg.LaplaceFMM(x, q, a)
    g.setup()
    rphi, rgrad = g.evaluate()
    assert np.array_equal(phi, rphi) and np.array_equal(grad, rgrad)
    # a second solve on the same handle with new charges
    q2 = np.random.default_rng(81).standard_normal(len(q))
    f.q = q2 - q2.mean()
    phi2, grad2 = f.solve()
    rphi2, rgrad2 = g.evaluate(f.q)
    assert np.array_equal(phi2, rphi2) and np.array_equal(grad2, rgrad2)
    f.close()
    g.close()
