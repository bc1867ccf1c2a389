"""The forward pass replayed as a CUDA graph.

Without RTFMM_STAGE_TIMED (and without RTFMM_STAGE_SERIAL) the library
captures the pass once per set of device tables and replays it.  The replay
must give bit-for-bit the outputs of the same launches issued directly, pick
up new charges and positions, and be rebuilt with the tables.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def uniform01(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 3))
    q = rng.random(n) * 2 - 1
    return x, q - q.mean()


def args(pkg, precision, stages, dipole=0):
    return pkg.Argument(P=6, ncrit=64, images=2, cycle=1.0, x=(0.5, 0.5, 0.5), dipole_correction=dipole,
                        divide_4pi=1, precision=precision, stages=stages)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("dipole", [0, 1])
def test_graph_replay_equals_direct_launches(pkg, precision, dipole):
    x, q = uniform01(20000, 31)
    g = pkg.LaplaceFMM(x, q, args(pkg, precision, pkg.STAGE_ALL, dipole))
    d = pkg.LaplaceFMM(x, q, args(pkg, precision, pkg.STAGE_ALL | pkg.STAGE_TIMED, dipole))
    for f in (g, d):
        f.setup()
        f.upload()
    for _ in range(3):  # capture, then two replays
        g.evaluate_device()
    d.evaluate_device()
    pg, gg = g.download()
    pd, gd = d.download()
    assert np.array_equal(pg, pd) and np.array_equal(gg, gd)
    assert all(v == 0 for v in g.stage_times().values())
    assert d.stage_times()["P2P"] > 0

    # new charges through the host call and through device buffers
    q2 = np.random.default_rng(32).standard_normal(len(q))
    p2g, g2g = g.evaluate(q2)
    p2d, g2d = d.evaluate(q2)
    assert np.array_equal(p2g, p2d) and np.array_equal(g2g, g2d)
    torch = pytest.importorskip("torch")
    q3 = torch.from_numpy(np.random.default_rng(33).standard_normal(len(q))).cuda()
    phi3 = torch.empty(len(q), dtype=torch.float64, device="cuda")
    grad3 = torch.empty((len(q), 3), dtype=torch.float64, device="cuda")
    g.forward_device(q3.data_ptr(), phi3.data_ptr(), grad3.data_ptr())
    p3d, g3d = d.evaluate(q3.cpu().numpy())
    assert np.array_equal(phi3.cpu().numpy(), p3d) and np.array_equal(grad3.cpu().numpy(), g3d)

    # new positions: new tables, new graph
    x4, q4 = uniform01(15000, 34)
    g4 = pkg.LaplaceFMM(x4, q4, args(pkg, precision, pkg.STAGE_ALL, dipole))
    d4 = pkg.LaplaceFMM(x4, q4, args(pkg, precision, pkg.STAGE_ALL | pkg.STAGE_TIMED, dipole))
    p4g, g4g = g4.solve()
    p4g2, g4g2 = g4.solve()  # a second solve on the same handle: re-setup, re-capture
    p4d, g4d = d4.solve()
    assert np.array_equal(p4g, p4d) and np.array_equal(g4g, g4d)
    assert np.array_equal(p4g2, p4d) and np.array_equal(g4g2, g4d)
    for f in (g, d, g4, d4):
        f.close()


def test_non_finite_charges_leave_the_handle_usable(pkg):
    """A non-finite charge is refused (checked while the charges are copied)
    and the next call with valid charges gives the same outputs as before."""
    x, q = uniform01(8000, 35)
    f = pkg.LaplaceFMM(x, q, args(pkg, 1, pkg.STAGE_ALL))
    p0, g0 = f.solve()
    bad = q.copy()
    bad[123] = np.nan
    with pytest.raises(pkg.RtfmmError) as e:
        f.evaluate(bad)
    assert e.value.code == 1
    p1, g1 = f.evaluate(q)
    assert np.array_equal(p0, p1) and np.array_equal(g0, g1)
    f.close()
