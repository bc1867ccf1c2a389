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


def setup_case(pkg, n, P, ncrit, seed):
    """An ordinary far-field FP64 pass and what the allocation-free call
    needs from its set-up: leaf records, tree-order bodies, U, (V S^-1)^T and
    the pass's leaf q_equiv."""
    rng = np.random.default_rng(seed)
    x = rng.random((n, 3))
    q = rng.random(n) * 2 - 1
    q -= q.mean()
    a = pkg.Argument(P=P, ncrit=ncrit, images=0, cycle=1.0, x=(0.5, 0.5, 0.5), dipole_correction=0, divide_4pi=1,
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
    f.close()
    return rec, bodies, U.copy(), VSinvT, q_equiv[leaves], ns


class Dev:
    def __init__(self, pkg, rec, bodies, U, VSinvT):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", 0)
        self.leaves = torch.from_numpy(rec.view(np.uint8).copy()).to(self.dev)
        self.bodies = torch.from_numpy(bodies).to(self.dev)
        self.U = torch.from_numpy(U).to(self.dev)
        self.VT = torch.from_numpy(VSinvT).to(self.dev)
        self.stream = torch.cuda.current_stream(self.dev).cuda_stream
        self.fn = bind(pkg)
        self.pkg = pkg

    def raw(self, P, nl, out_ptr, bodies_ptr=None):
        return self.fn(P, nl, self.leaves.data_ptr(), bodies_ptr or self.bodies.data_ptr(), self.U.data_ptr(),
                       self.VT.data_ptr(), out_ptr, self.stream)

    def call(self, P, nl, ns):
        out = self.torch.full((nl, ns), float("nan"), dtype=self.torch.float64, device=self.dev)
        rc = self.raw(P, nl, out.data_ptr())
        assert rc == 0, self.pkg.lib().rtfmm_b200_last_error()
        self.torch.cuda.synchronize(self.dev)
        return out.cpu().numpy()


def test_p2m_noalloc_matches_pass(pkg):
    P = 6
    rec, bodies, U, VSinvT, ref, ns = setup_case(pkg, 4000, P, 32, 11)
    d = Dev(pkg, rec, bodies, U, VSinvT)
    scale = np.abs(ref).max()
    # two calls in a row: all leaves, then the first half into a fresh buffer
    out1 = d.call(P, len(rec), ns)
    assert np.abs(out1 - ref).max() / scale < 1e-12
    half = len(rec) // 2
    out2 = d.call(P, half, ns)
    assert np.abs(out2 - ref[:half]).max() / scale < 1e-12

    # a batch larger than the fixed scratch is refused before any launch, and
    # so is a count whose size arithmetic would wrap
    for nl in (1 << 20, 1 << 62):
        rc = d.raw(8, nl, d.bodies.data_ptr())
        assert rc == 1 and b"scratch" in pkg.lib().rtfmm_b200_last_error()
    # misaligned caller buffers are refused (8-byte offsets into the bodies
    # and into an output buffer)
    out = d.torch.zeros(len(rec) * ns + 2, dtype=d.torch.float64, device=d.dev)
    rc = d.raw(P, len(rec), out.data_ptr(), bodies_ptr=d.bodies.data_ptr() + 8)
    assert rc == 1 and b"aligned" in pkg.lib().rtfmm_b200_last_error()
    rc = d.raw(P, len(rec), out.data_ptr() + 8)
    assert rc == 1 and b"aligned" in pkg.lib().rtfmm_b200_last_error()
    # the refusals left the output untouched
    d.torch.cuda.synchronize(d.dev)
    assert float(out.abs().max()) == 0.0


def test_p2m_noalloc_largest_batch_p8(pkg):
    """At P = 8 the scratch holds 1765 leaves: that batch runs and matches
    the pass (the scratch used to within 159 doubles of its end), and 1766
    leaves are refused."""
    P = 8
    rec, bodies, U, VSinvT, ref, ns = setup_case(pkg, 60000, P, 32, 12)
    assert ns == 296 and len(rec) > 1766
    d = Dev(pkg, rec, bodies, U, VSinvT)
    scale = np.abs(ref).max()
    out = d.call(P, 1765, ns)
    assert np.abs(out - ref[:1765]).max() / scale < 1e-12
    rc = d.raw(P, 1766, d.bodies.data_ptr())
    assert rc == 1 and b"scratch" in pkg.lib().rtfmm_b200_last_error()
    # a second call in a row on the same scratch: the last 1765 leaves
    tail = Dev(pkg, rec[-1765:].copy(), bodies, U, VSinvT)
    out = tail.call(P, 1765, ns)
    assert np.abs(out - ref[-1765:]).max() / scale < 1e-12
