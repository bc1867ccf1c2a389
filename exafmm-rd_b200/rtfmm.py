"""Python mirror of the reference's FMM driver interface, over the C ABI.

The reference (mumairsadiq/exafmm-rd, variant 3dpp) is driven as

    Argument args(argc, argv);                    // 3dpp/src/argument.cpp:7-70
    Bodies3 bs = generate_random_bodies(...);     // 3dpp/src/body.cpp:98-129
    Bodies3 res = LaplaceFMM(bs, args).solve();   // 3dpp/src/fmm.cpp:13-81
    compare(res, ref, ...).show();                // 3dpp/src/body.cpp:131-205

This module keeps those names and meanings.  Bodies are passed as numpy
arrays (positions (n,3), charges (n,)); results come back in input order as
(potential (n,), gradient (n,3)), the reference's Body3::p and Body3::f.

All arithmetic runs in librtfmm_b200.so (CUDA kernels for sm_100a and the
host set-up in C++).  There is no CPU fallback: if the library is missing or
no GPU is visible, the evaluation raises.
"""
import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librtfmm_b200.so")

RTFMM_OK, RTFMM_EINVAL, RTFMM_ENOMEM, RTFMM_ECUDA, RTFMM_ESTATE, RTFMM_ENOTSUP, RTFMM_ETIMEOUT = range(7)
FP64, FP32_MIXED = 0, 1
STAGE_NEAR, STAGE_FAR, STAGE_ALL, STAGE_SERIAL, STAGE_TIMED = 1, 2, 3, 4, 8
STAGE_NAMES = ("prep", "P2M", "M2M", "M2L_up", "M2L_hadamard", "M2L_down", "L2L", "L2P", "P2P", "post")

# Every entry point declared in include/rtfmm_b200.h.
EXPORTS = (
    "rtfmm_b200_default_args", "rtfmm_b200_create", "rtfmm_b200_destroy", "rtfmm_b200_setup",
    "rtfmm_b200_setup_device",
    "rtfmm_b200_evaluate", "rtfmm_b200_solve", "rtfmm_b200_upload", "rtfmm_b200_evaluate_device",
    "rtfmm_b200_download", "rtfmm_b200_forward_device", "rtfmm_b200_adjoint", "rtfmm_b200_adjoint_device",
    "rtfmm_b200_stage_times",
    "rtfmm_b200_launch_count",
    "rtfmm_b200_flush_l2", "rtfmm_b200_setup_times", "rtfmm_b200_info", "rtfmm_b200_get_cells", "rtfmm_b200_get_perm",
    "rtfmm_b200_get_p2p", "rtfmm_b200_get_m2l", "rtfmm_b200_get_leaf_lists", "rtfmm_b200_get_cell_vectors", "rtfmm_b200_get_operator",
    "rtfmm_b200_last_error", "rtfmm_b200_version", "rtfmm_b200_clear_operator_cache",
    "rtfmm_b200_save_operators", "rtfmm_b200_load_operators", "rtfmm_b200_p2m_noalloc",
    "rtfmm_b200_ewald_sampled", "rtfmm_b200_direct_sampled",
    "rtfmm_b200_shard", "rtfmm_b200_shard_sizes", "rtfmm_b200_shard_bodies", "rtfmm_b200_shard_upward",
    "rtfmm_b200_shard_downward",
)


class RtfmmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("rtfmm_b200 error %d: %s" % (code, msg))
        self.code = code


class _Args(ctypes.Structure):
    _fields_ = [("P", ctypes.c_int), ("ncrit", ctypes.c_int), ("images", ctypes.c_int),
                ("cycle", ctypes.c_double), ("x", ctypes.c_double * 3),
                ("dipole_correction", ctypes.c_int), ("divide_4pi", ctypes.c_int),
                ("precision", ctypes.c_int), ("stages", ctypes.c_uint), ("device", ctypes.c_int)]


_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_lp = ctypes.POINTER(ctypes.c_int64)
_fp = ctypes.POINTER(ctypes.c_float)
_vp = ctypes.c_void_p


def lib():
    """Loads librtfmm_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RtfmmError(RTFMM_ENOTSUP, "librtfmm_b200.so not built (run exafmm-rd_b200/build.py)")
    L = ctypes.CDLL(LIB_PATH)
    sig = {
        "rtfmm_b200_default_args": (None, [ctypes.POINTER(_Args)]),
        "rtfmm_b200_create": (ctypes.c_int, [ctypes.POINTER(_Args), ctypes.POINTER(_vp)]),
        "rtfmm_b200_destroy": (ctypes.c_int, [_vp]),
        "rtfmm_b200_setup": (ctypes.c_int, [_vp, ctypes.c_int64, _dp, _dp]),
        "rtfmm_b200_setup_device": (ctypes.c_int, [_vp, ctypes.c_int64, _vp, _vp]),
        "rtfmm_b200_evaluate": (ctypes.c_int, [_vp, _dp, _dp, _dp]),
        "rtfmm_b200_solve": (ctypes.c_int, [_vp, ctypes.c_int64, _dp, _dp, _dp, _dp]),
        "rtfmm_b200_upload": (ctypes.c_int, [_vp]),
        "rtfmm_b200_evaluate_device": (ctypes.c_int, [_vp, _fp]),
        "rtfmm_b200_download": (ctypes.c_int, [_vp, _dp, _dp]),
        "rtfmm_b200_adjoint": (ctypes.c_int, [_vp, _dp, _dp, _dp]),
        "rtfmm_b200_adjoint_device": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_float)]),
        "rtfmm_b200_forward_device": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_float)]),
        "rtfmm_b200_ewald_sampled": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, _dp, _dp, ctypes.c_double,
                                                    ctypes.c_int, ctypes.c_int64, _lp, _dp, _dp]),
        "rtfmm_b200_direct_sampled": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, _dp, _dp, ctypes.c_int64, _lp,
                                                     _dp, _dp]),
        "rtfmm_b200_stage_times": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
        "rtfmm_b200_launch_count": (ctypes.c_int, [_vp, _lp]),
        "rtfmm_b200_flush_l2": (ctypes.c_int, [_vp]),
        "rtfmm_b200_info": (ctypes.c_int, [_vp, _lp, ctypes.c_int]),
        "rtfmm_b200_setup_times": (ctypes.c_int, [_vp, _dp, ctypes.c_int]),
        "rtfmm_b200_clear_operator_cache": (None, []),
        "rtfmm_b200_save_operators": (ctypes.c_int, [_vp, ctypes.c_char_p]),
        "rtfmm_b200_load_operators": (ctypes.c_int, [ctypes.c_char_p]),
        "rtfmm_b200_get_cells": (ctypes.c_int, [_vp, _ip, _dp]),
        "rtfmm_b200_get_perm": (ctypes.c_int, [_vp, _lp]),
        "rtfmm_b200_get_p2p": (ctypes.c_int, [_vp, _ip, _dp]),
        "rtfmm_b200_get_m2l": (ctypes.c_int, [_vp, _ip, _dp]),
        "rtfmm_b200_get_cell_vectors": (ctypes.c_int, [_vp, ctypes.c_int, _dp]),
        "rtfmm_b200_get_operator": (ctypes.c_int, [_vp, ctypes.c_int, _dp, ctypes.c_int64]),
        "rtfmm_b200_get_leaf_lists": (ctypes.c_int, [_vp, _ip, _ip, _dp, ctypes.c_int64]),
        "rtfmm_b200_shard": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
        "rtfmm_b200_shard_sizes": (ctypes.c_int, [_vp, _lp, _lp]),
        "rtfmm_b200_shard_bodies": (ctypes.c_int, [_vp, _lp, ctypes.c_int64]),
        "rtfmm_b200_shard_upward": (ctypes.c_int, [_vp, _vp]),
        "rtfmm_b200_shard_downward": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.POINTER(ctypes.c_float)]),
        "rtfmm_b200_last_error": (ctypes.c_char_p, []),
        "rtfmm_b200_version": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def _check(rc):
    if rc != RTFMM_OK:
        raise RtfmmError(rc, lib().rtfmm_b200_last_error().decode())
    return rc


def _ptr(a, typ=_dp):
    return a.ctypes.data_as(typ) if a is not None else None


class Argument:
    """Run parameters with the names of rtfmm::Argument
    (3dpp/include/argument.h:11-45).  Defaults follow argument.cpp:11-31;
    ``r`` is cycle/2 and ``x`` is the box centre (argument.cpp:61-62).
    ``setting_t`` applies the reference's override (argument.cpp:64-69)."""

    def __init__(self, P=4, n=1000, ncrit=16, images=0, cycle=2 * math.pi, seed=5,
                 dipole_correction=1, zero_netcharge=1, divide_4pi=0, setting_t=0,
                 x=(0.0, 0.0, 0.0), precision=FP64, stages=STAGE_ALL, device=0, num_compare=-1,
                 ewald_ksize=11):
        self.P = P
        self.n = n
        self.ncrit = ncrit
        self.images = images
        self.cycle = cycle
        self.seed = seed
        self.dipole_correction = dipole_correction
        self.zero_netcharge = zero_netcharge
        self.divide_4pi = divide_4pi
        self.setting_t = setting_t
        self.x = tuple(x)
        self.precision = precision
        self.stages = stages
        self.device = device
        self.num_compare = n if num_compare == -1 else num_compare
        self.ewald_ksize = ewald_ksize
        if setting_t:
            self.dipole_correction = 0
            self.zero_netcharge = 0
            self.divide_4pi = 1

    @property
    def r(self):
        return self.cycle / 2

    def _c(self):
        a = _Args()
        lib().rtfmm_b200_default_args(ctypes.byref(a))
        a.P, a.ncrit, a.images, a.cycle = self.P, self.ncrit, self.images, self.cycle
        for k in range(3):
            a.x[k] = self.x[k]
        # 0 / 1 as the reference's flag; 2 the surface term's potential
        a.dipole_correction = int(self.dipole_correction) if self.dipole_correction in (0, 1, 2) else 1
        a.divide_4pi = int(bool(self.divide_4pi))
        a.precision = self.precision
        a.stages = self.stages
        a.device = self.device
        return a


class LaplaceFMM:
    """``rtfmm::LaplaceFMM`` (3dpp/include/fmm.h:12-45): construct with the
    bodies and the arguments, then ``solve()``.

    ``x`` is (n,3) and ``q`` is (n,), float64.  ``solve()`` returns the
    potential (n,) and its gradient (n,3) in input order."""

    def __init__(self, x, q, args):
        self.args = args
        self.x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 3)
        self.q = np.ascontiguousarray(q, dtype=np.float64).reshape(-1)
        if self.x.shape[0] != self.q.shape[0]:
            raise RtfmmError(RTFMM_EINVAL, "LaplaceFMM init body size error")
        self.n = self.q.shape[0]
        h = _vp()
        ca = args._c()
        _check(lib().rtfmm_b200_create(ctypes.byref(ca), ctypes.byref(h)))
        self._h = h
        self._set_up = False

    def close(self):
        if getattr(self, "_h", None):
            lib().rtfmm_b200_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- phases ---------------------------------------------------------------
    def setup(self):
        """Tree, lists and operator tables (host; fmm.cpp:15-49)."""
        _check(lib().rtfmm_b200_setup(self._h, self.n, _ptr(self.x), _ptr(self.q)))
        self._set_up = True

    def setup_device(self, x_ptr, q_ptr, n=None):
        """Set-up from bodies in device memory: integer device addresses
        (e.g. a torch tensor's data_ptr()) of x (n, 3) and q (n), float64.
        The octree is built on the GPU; the bodies stay on the device, so
        evaluate_device() / forward_device() follow without upload()."""
        n = self.n if n is None else int(n)
        _check(lib().rtfmm_b200_setup_device(self._h, n, _vp(x_ptr or None), _vp(q_ptr or None)))
        self.n = n
        self._set_up = True

    def evaluate(self, q=None):
        """The evaluation pass with host buffers; returns (phi, grad)."""
        if not self._set_up:
            self.setup()
        phi = np.empty(self.n)
        grad = np.empty((self.n, 3))
        qq = None if q is None else np.ascontiguousarray(q, dtype=np.float64)
        _check(lib().rtfmm_b200_evaluate(self._h, _ptr(qq), _ptr(phi), _ptr(grad)))
        return phi, grad

    def solve(self):
        """``LaplaceFMM::solve`` (fmm.cpp:13-81): rtfmm_b200_solve (set-up on
        the GPU from 65536 bodies, else on the host; the same plan), then the
        pass."""
        phi = np.empty(self.n)
        grad = np.empty((self.n, 3))
        _check(lib().rtfmm_b200_solve(self._h, self.n, _ptr(self.x), _ptr(self.q), _ptr(phi), _ptr(grad)))
        self._set_up = True
        return phi, grad

    # -- device-resident timing -------------------------------------------------
    def upload(self):
        _check(lib().rtfmm_b200_upload(self._h))

    def evaluate_device(self):
        ms = ctypes.c_float(0)
        _check(lib().rtfmm_b200_evaluate_device(self._h, ctypes.byref(ms)))
        return ms.value

    def download(self):
        phi = np.empty(self.n)
        grad = np.empty((self.n, 3))
        _check(lib().rtfmm_b200_download(self._h, _ptr(phi), _ptr(grad)))
        return phi, grad

    def flush_l2(self):
        _check(lib().rtfmm_b200_flush_l2(self._h))

    def stage_times(self):
        v = np.zeros(len(STAGE_NAMES))
        lib().rtfmm_b200_stage_times(self._h, _ptr(v), len(v))
        return dict(zip(STAGE_NAMES, v.tolist()))

    def launch_count(self):
        v = ctypes.c_int64(0)
        _check(lib().rtfmm_b200_launch_count(self._h, ctypes.byref(v)))
        return v.value

    def adjoint(self, w):
        w = np.ascontiguousarray(w, dtype=np.float64)
        dq = np.empty(self.n)
        dx = np.empty((self.n, 3))
        _check(lib().rtfmm_b200_adjoint(self._h, _ptr(w), _ptr(dq), _ptr(dx)))
        return dq, dx

    def forward_device(self, q_ptr, phi_ptr, grad_ptr):
        """The pass on device memory: integer device addresses of q (n, or 0
        to keep the charges on the device), phi (n) and grad (n, 3), input
        order, float64.  Returns the pass time in ms."""
        ms = ctypes.c_float(0)
        _check(lib().rtfmm_b200_forward_device(self._h, _vp(q_ptr or None), _vp(phi_ptr or None),
                                               _vp(grad_ptr or None), ctypes.byref(ms)))
        return ms.value

    def adjoint_device(self, w_ptr, dq_ptr, dx_ptr):
        """Adjoint on device memory: integer device addresses (e.g. a torch
        tensor's data_ptr()) of w (n), dL/dq (n) and dL/dx (n, 3), input
        order, float64.  Returns the device time in ms."""
        ms = ctypes.c_float(0)
        _check(lib().rtfmm_b200_adjoint_device(self._h, _vp(w_ptr), _vp(dq_ptr or None), _vp(dx_ptr or None),
                                               ctypes.byref(ms)))
        return ms.value

    # -- the pass sharded over ranks ------------------------------------------------
    def shard(self, rank, nranks):
        """This handle computes rank `rank` of `nranks` shares of the pass
        (before setup(); see rtfmm_b200_shard in include/rtfmm_b200.h)."""
        _check(lib().rtfmm_b200_shard(self._h, int(rank), int(nranks)))
        self._set_up = False

    def shard_sizes(self):
        """(bodies computed by this rank, doubles of the exchange buffer)."""
        nb, nx = ctypes.c_int64(0), ctypes.c_int64(0)
        _check(lib().rtfmm_b200_shard_sizes(self._h, ctypes.byref(nb), ctypes.byref(nx)))
        return nb.value, nx.value

    def shard_bodies(self):
        """Input indices of the bodies whose outputs this rank computes."""
        nb, _ = self.shard_sizes()
        idx = np.zeros(max(nb, 1), dtype=np.int64)
        _check(lib().rtfmm_b200_shard_bodies(self._h, _ptr(idx, _lp), nb))
        return idx[:nb]

    def shard_upward(self, xbuf_ptr):
        """P2M of this rank's leaves; every leaf's q_equiv row into the device
        buffer at xbuf_ptr (others' rows zero), to be summed over the ranks."""
        _check(lib().rtfmm_b200_shard_upward(self._h, _vp(xbuf_ptr)))

    def shard_downward(self, xbuf_ptr, phi_ptr, grad_ptr):
        """The rest of the pass from the summed buffer; this rank's outputs
        into the device arrays at phi_ptr (n) and grad_ptr (n, 3).  Returns
        the device time of this phase in ms."""
        ms = ctypes.c_float(0)
        _check(lib().rtfmm_b200_shard_downward(self._h, _vp(xbuf_ptr), _vp(phi_ptr or None),
                                               _vp(grad_ptr or None), ctypes.byref(ms)))
        return ms.value

    # -- introspection ------------------------------------------------------------
    def save_operators(self, path):
        """Writes this handle's operator tables to `path` (after setup)."""
        _check(lib().rtfmm_b200_save_operators(self._h, os.fsencode(path)))

    def setup_times(self):
        """Wall seconds of the last set-up's phases: tree, lists, operators
        (0 when cached), host tables, the setup call, and the upload of the
        device tables; then the operator build's parts (0 when cached): SVD,
        Gram-Schmidt, M2M products, image products, kernel spectra, blocks."""
        v = np.zeros(12)
        _check(lib().rtfmm_b200_setup_times(self._h, _ptr(v), 12))
        return dict(zip(("tree", "lists", "operators", "tables", "total", "upload", "ops_svd", "ops_orth",
                         "ops_m2m", "ops_img", "ops_spectra", "ops_blocks"), v.tolist()))

    def info(self):
        v = np.zeros(13, dtype=np.int64)
        lib().rtfmm_b200_info(self._h, _ptr(v, _lp), 13)
        keys = ("ncell", "nleaf", "depth_min", "depth_max", "n_p2p", "n_m2l_parents", "n_m2l", "num_surf",
                "p2p_pairs", "m2l8_pairs", "m2l8_sources", "m2l8_targets", "close_pairs")
        return dict(zip(keys, v.tolist()))

    def cells(self):
        nc = self.info()["ncell"]
        ints = np.zeros((nc, 7), dtype=np.int32)
        reals = np.zeros((nc, 4))
        _check(lib().rtfmm_b200_get_cells(self._h, _ptr(ints, _ip), _ptr(reals)))
        return ints, reals

    def perm(self):
        p = np.zeros(self.n, dtype=np.int64)
        _check(lib().rtfmm_b200_get_perm(self._h, _ptr(p, _lp)))
        return p

    def p2p_lists(self):
        m = self.info()["n_p2p"]
        ints = np.zeros((m, 2), dtype=np.int32)
        off = np.zeros((m, 3))
        _check(lib().rtfmm_b200_get_p2p(self._h, _ptr(ints, _ip), _ptr(off)))
        return ints, off

    def leaf_lists(self):
        """The pass's P2P lists by target leaf: (list_off, src_leaf, off)."""
        nleaf = self.info()["nleaf"]
        lo = np.zeros(nleaf + 1, dtype=np.int32)
        _check(lib().rtfmm_b200_get_leaf_lists(self._h, _ptr(lo, _ip), None, None, 0))
        m = int(lo[-1])
        src = np.zeros(max(m, 1), dtype=np.int32)
        off = np.zeros((max(m, 1), 3))
        _check(lib().rtfmm_b200_get_leaf_lists(self._h, _ptr(lo, _ip), _ptr(src, _ip), _ptr(off), m))
        return lo, src[:m], off[:m]

    def m2l_lists(self):
        m = self.info()["n_m2l"]
        ints = np.zeros((m, 3), dtype=np.int32)
        off = np.zeros((m, 3))
        _check(lib().rtfmm_b200_get_m2l(self._h, _ptr(ints, _ip), _ptr(off)))
        return ints, off

    def cell_vectors(self, which):
        inf = self.info()
        out = np.zeros((inf["ncell"], inf["num_surf"]))
        _check(lib().rtfmm_b200_get_cell_vectors(self._h, which, _ptr(out)))
        return out

    def operator(self, which, size):
        out = np.zeros(size)
        _check(lib().rtfmm_b200_get_operator(self._h, which, _ptr(out), size))
        return out


# ----------------------------------------------------------------------------
# bodies and the comparison metric
# ----------------------------------------------------------------------------
def load_operators(path):
    """Loads operator tables saved by LaplaceFMM.save_operators into the
    process-wide cache (set-ups with the same P, images and cycle use them)."""
    _check(lib().rtfmm_b200_load_operators(os.fsencode(path)))


def clear_operator_cache():
    """Frees the process-wide cache of operator tables that handles with the
    same (P, images, cycle) share; the next set-up builds its tables."""
    lib().rtfmm_b200_clear_operator_cache()


def drand48_stream(seed, count):
    """glibc srand48/drand48: 48-bit LCG, a = 0x5DEECE66D, c = 0xB, state
    (seed << 16) | 0x330E; returns ``count`` doubles state / 2^48."""
    a, c, m = 0x5DEECE66D, 0xB, (1 << 48) - 1
    x = ((seed & 0xFFFFFFFF) << 16) | 0x330E
    out = np.empty(count)
    for i in range(count):
        x = (a * x + c) & m
        out[i] = x / float(1 << 48)
    return out


def generate_random_bodies(n, r, offset=(0.0, 0.0, 0.0), seed=5, zero_netcharge=1):
    """``generate_random_bodies`` (3dpp/src/body.cpp:98-129)."""
    u = drand48_stream(seed, 4 * n).reshape(n, 4)
    x = u[:, :3] * r * 2 - r + np.asarray(offset, dtype=np.float64)
    q = u[:, 3] - 0.5
    if zero_netcharge and n:
        q = q - (sum(q.tolist()) / n)
    return x, q


def ewald_sampled(x, q, cycle, targets, ksize=11, device=0):
    """Ewald sum on sampled targets, FP64 on the GPU (EwaldSolver,
    3dpp/src/ewald.cpp): (phi, grad) at bodies ``targets``, no 1/(4 pi)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    phi = np.empty(len(t))
    grad = np.empty((len(t), 3))
    _check(lib().rtfmm_b200_ewald_sampled(device, len(q), _ptr(x), _ptr(q), float(cycle), int(ksize), len(t),
                                          _ptr(t, _lp), _ptr(phi), _ptr(grad)))
    return phi, grad


def direct_sampled(x, q, targets, device=0):
    """Free-space direct sum on sampled targets, FP64 on the GPU: (phi, grad)
    at bodies ``targets``, no 1/(4 pi)."""
    x = np.ascontiguousarray(x, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    phi = np.empty(len(t))
    grad = np.empty((len(t), 3))
    _check(lib().rtfmm_b200_direct_sampled(device, len(q), _ptr(x), _ptr(q), len(t), _ptr(t, _lp), _ptr(phi),
                                           _ptr(grad)))
    return phi, grad


def compare(p1, f1, q1, p2, f2, q2):
    """``compare`` (3dpp/src/body.cpp:131-175); the second set is the norm."""
    p1, p2 = np.asarray(p1), np.asarray(p2)
    f1, f2 = np.asarray(f1).reshape(-1, 3), np.asarray(f2).reshape(-1, 3)
    pdif = float(np.sum((p1 - p2) ** 2))
    pnrm = float(np.sum(p2 ** 2))
    fdif = float(np.sum((f1 - f2) ** 2))
    fnrm = float(np.sum(f2 ** 2))
    e1 = float(np.sum(p1 * q1))
    e2 = float(np.sum(p2 * q2))
    n = len(p1)
    return {"l2p": math.sqrt(pdif / pnrm) if pnrm else float("nan"),
            "l2f": math.sqrt(fdif / fnrm) if fnrm else float("nan"),
            "l2e": abs(e1 - e2) / abs(e2) if e2 else float("nan"),
            "rmsp": math.sqrt(pdif / n) if n else 0.0, "rmsf": math.sqrt(fdif / n) if n else 0.0,
            "energy1": e1, "energy2": e2}
