"""The allocation-free P2M entry point, checked against the evaluation pass.

Code that runs under another framework's device-memory pool cannot call
cudaMalloc itself: an allocation outside the pool would escape its
accounting or fail against its limits.  rtfmm_b200_p2m_noalloc gives such
callers the P2M stage with its scratch in a fixed array inside the library;
they pass only their own input and output buffers.  Its output must equal
the leaf equivalent densities of the ordinary evaluation pass, call after
call.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LEAF = np.dtype([("cx", "f8"), ("cy", "f8"), ("cz", "f8"), ("r", "f8"), ("scale", "f8"), ("cell", "i4"),
                 ("boff", "i4"), ("bnum", "i4"), ("pad", "i4")])


def bind(pkg):
    fn = pkg.lib().rtfmm_b200_p2m_noalloc
    fn.restype = ctypes.c_int
    fn.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return fn


def test_p2m_noalloc_matches_pass(pkg):
    import torch
    rng = np.random.default_rng(11)
    n, P = 4000, 6
    x = rng.random((n, 3))
    q = rng.random(n) * 2 - 1
    q -= q.mean()
    # the ordinary entry point: far field only, FP64, then its leaf q_equiv
    a = pkg.Argument(P=P, ncrit=32, images=0, cycle=1.0, x=(0.5, 0.5, 0.5), dipole_correction=0, divide_4pi=1,
                     precision=pkg.FP64, stages=pkg.STAGE_FAR)
    f = pkg.LaplaceFMM(x, q, a)
    f.solve()
    q_equiv = f.cell_vectors(0)
    info = f.info()
    ns = info["num_surf"]
    ints, reals = f.cells()
    leaves = [c for c in range(info["ncell"]) if ints[c, 3] == 0 and ints[c, 1] >= 0]
    rec = np.zeros(len(leaves), dtype=LEAF)
    for i, c in enumerate(leaves):
        rec[i] = (reals[c, 1], reals[c, 2], reals[c, 3], reals[c, 0], 0.5 ** int(ints[c, 1]), c,
                  ints[c, 4], ints[c, 5], 0)
    perm = f.perm()
    bodies = np.ascontiguousarray(np.concatenate([x[perm], q[perm][:, None]], axis=1))
    U = f.operator(4, ns * ns).reshape(ns, ns)
    VSinvT = np.ascontiguousarray(f.operator(5, ns * ns).reshape(ns, ns).T)
    ref = q_equiv[leaves]

    dev = torch.device("cuda", 0)
    d_leaves = torch.from_numpy(rec.view(np.uint8).copy()).to(dev)
    d_bodies = torch.from_numpy(bodies).to(dev)
    d_U = torch.from_numpy(U.copy()).to(dev)
    d_VT = torch.from_numpy(VSinvT).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    fn = bind(pkg)

    def call(nl, out):
        rc = fn(P, nl, d_leaves.data_ptr(), d_bodies.data_ptr(), d_U.data_ptr(), d_VT.data_ptr(),
                out.data_ptr(), stream)
        assert rc == 0, pkg.lib().rtfmm_b200_last_error()
        torch.cuda.synchronize(dev)
        return out.cpu().numpy()

    scale = np.abs(ref).max()
    # two calls in a row: all leaves, then the first half into a fresh buffer
    out1 = call(len(leaves), torch.full((len(leaves), ns), np.nan, dtype=torch.float64, device=dev))
    assert np.abs(out1 - ref).max() / scale < 1e-12
    half = len(leaves) // 2
    out2 = call(half, torch.full((half, ns), np.nan, dtype=torch.float64, device=dev))
    assert np.abs(out2 - ref[:half]).max() / scale < 1e-12

    # a batch larger than the fixed scratch is refused before any launch
    rc = fn(8, 1 << 20, d_leaves.data_ptr(), d_bodies.data_ptr(), d_U.data_ptr(), d_VT.data_ptr(),
            d_bodies.data_ptr(), stream)
    assert rc == 1 and b"scratch" in pkg.lib().rtfmm_b200_last_error()
