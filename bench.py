"""Throughput of the periodic KIFMM evaluation pass on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (the configuration the headline metric is quoted on): N = 2^20
bodies i.i.d. uniform in [0,1)^3, charges uniform in [-1,1] shifted to zero
net charge (seed 2), P = 8, ncrit = 256, 3 periodic image levels, cycle 1,
kernel 1/(4 pi r), no dipole correction.  A step is one evaluation pass
(the reference's FMM_kernels block: P2M, M2M, M2L, L2L, L2P, P2P, then the
1/(4 pi) scaling and the re-sort), with the octree, lists and operator
tables built beforehand, as the reference times it.

ours:       value = N / pass time, FP32-mixed form, bodies resident in HBM,
            256 MB L2 flush between steps; the FP64 form of the same pass is
            timed beside it and its error against the FP64 form is reported.
            e2e   = the same metric through the C ABI with pinned host
            buffers (charges in, potential and gradient out) per step.
reference:  the reference's own CPU FMM (compiled from its sources into
            oracle/_ref, else the numpy oracle) on the same workload, all
            host threads: its tree, lists and tables built once, then one
            run of its hot block per step.

Multi-GPU (torchrun): by default each rank runs an independent replica on
its own GPU; value = all ranks' bodies / max-over-ranks time.  With --shard
the ranks split one pass (rtfmm_b200_shard: each computes its share of the
bodies; one NCCL all-reduce of the leaf q_equiv rows per pass).
"""
import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "particles/s potential+force, N=1M P=8 PBC: FP32-mixed vs FP64 GPU at equal err"
WORKLOAD = dict(N=1 << 20, P=8, ncrit=256, images=3, cycle=1.0, seed=2)


def load_pkg():
    import importlib.util
    d = os.path.join(ROOT, "exafmm-rd_b200")
    spec = importlib.util.spec_from_file_location("exafmm_rd_b200", os.path.join(d, "__init__.py"),
                                                  submodule_search_locations=[d])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["exafmm_rd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def pass_roofline(info, n, Nf, had_flop, had_bytes, fp32_peak, sm_mhz, hbm, hbm_kind, pass_ms):
    """The whole pass against its roofline: each stage's algorithmic work
    (flops and bytes per unit as the scope table counts them) gives the time
    its bound allows, max(flops / compute peak, bytes / HBM peak); their sum
    over the measured pass time is the fraction of the roofline the pass
    reaches.  P2P and the Hadamard count against FP32, the operator stages
    against FP64 (nominal 148 SM x 64 FMA/clk x 2 at the sampled clock)."""
    ns, nl, N = info["num_surf"], info["nleaf"], n
    nch = max(info["ncell"] - 1, 0)  # every cell but the root is a child
    nsrc, ntar = info["m2l8_sources"], info["m2l8_targets"]
    fp64_peak = 148 * 64 * 2 * sm_mhz * 1e6 / 1e12
    bw = hbm * 1e9

    def bound(flop, peak_tf, nbytes):
        return max(flop / (peak_tf * 1e12), nbytes / bw)

    st = {
        # 20 flop per body pair; bodies read (16 B) and phi, grad written (32 B)
        "P2P": bound(20.0 * info["p2p_pairs"], fp32_peak, 48.0 * N),
        # 11 flop per body x check point, two ns x ns products per leaf
        "P2M": bound(11.0 * N * ns + 4.0 * ns * ns * nl, fp64_peak, 16.0 * N + 8.0 * ns * nl),
        "M2M": bound(2.0 * ns * ns * nch, fp64_peak, 16.0 * ns * nch),
        "M2L_up": bound(0.0, fp32_peak, (8.0 * ns * 8 + 8.0 * Nf * 8) * nsrc),
        "M2L_hadamard": bound(had_flop, fp32_peak, had_bytes),
        "M2L_down": bound(0.0, fp32_peak, (8.0 * ns * 8 + 8.0 * Nf * 8) * ntar),
        "L2L": bound(2.0 * ns * ns * nch, fp64_peak, 16.0 * ns * nch),
        # 20 flop per body x equivalent point, two products per leaf; bodies
        # read, phi and grad written
        "L2P": bound(20.0 * N * ns + 4.0 * ns * ns * nl, fp64_peak, 48.0 * N + 8.0 * ns * nl),
    }
    total = sum(st.values())
    return {"bound_ms": total * 1e3, "pass_ms": pass_ms, "frac": total * 1e3 / pass_ms,
            "stages_bound_ms": {k: v * 1e3 for k, v in st.items()},
            "peaks": {"fp32_tflops": fp32_peak, "fp64_tflops": fp64_peak, "hbm_gbs": hbm,
                      "kind": "FP32/FP64 nominal at the sampled SM clock; HBM " + hbm_kind}}


def make_bodies(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 3))
    q = rng.random(n) * 2 - 1
    return x, q - q.mean()


class ClockSampler:
    """SM clock and throttle reasons sampled through NVML (read-only) every
    10 ms during the timed region."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
               "sw_power_cap": 0x4}

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = nv.nvmlDeviceGetHandleByIndex(self.index)
            mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            while not self._stop.is_set():
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.samples.append((sm, mx, rs))
                self._stop.wait(0.01)
            nv.nvmlShutdown()
        except Exception:
            pass

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        reasons = sorted({nm for (_, _, r) in self.samples for nm, bit in self.REASONS.items() if r & bit})
        return {"sm_mhz": float(np.median([s[0] for s in self.samples])),
                "sm_max_mhz": float(max(s[1] for s in self.samples)), "reasons": reasons,
                "samples": len(self.samples)}


def read_traffic(kernel):
    """dram bytes per launch of the default workload, from the committed ncu
    summary, if present."""
    path = os.path.join(ROOT, "profiles", "k_%s_n1M_p8_traffic.txt" % kernel)
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("traffic_bytes_per_launch:"):
            return float(line.split(":", 1)[1])
    return None


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


# ----------------------------------------------------------------------------
# reference arm / CPU baseline
# ----------------------------------------------------------------------------
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "rtfmm_ref_pass")


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_passes(n, threads, passes, seed=2):
    """The reference's own CPU FMM on n bodies of the workload: its tree,
    lists and operator tables built once, then `passes` runs of its hot block
    (LaplaceFMM's P2M ... P2P, 3dpp/src/fmm.cpp:51-60; oracle/_ref
    rtfmm_ref_pass --repeat).  Returns (pass seconds list, set-up seconds,
    kind, note); without the compiled reference, the numpy oracle's whole
    pass (single process) instead."""
    W = WORKLOAD
    x, q = make_bodies(n, seed)
    if os.path.exists(REF_BIN):
        with tempfile.TemporaryDirectory() as td:
            fin = os.path.join(td, "in.bin")
            np.concatenate([x - 0.5, q[:, None]], axis=1).astype(np.float64).tofile(fin)
            env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS=str(threads))
            cmd = [REF_BIN, "--in", fin, "--repeat", str(passes), "-n", str(n), "-P", str(W["P"]),
                   "-m", str(W["ncrit"]), "-i", str(W["images"]), "-c", str(W["cycle"]), "--th_num", str(threads),
                   "--dipole_correction", "0", "--divide_4pi", "1"]
            out = subprocess.run(cmd, capture_output=True, text=True, env=env, timeout=3600).stdout
        ts, setup = [], None
        for line in out.splitlines():
            if line.startswith("[repeat_pass"):
                ts.append(float(line.split()[2]))
            elif line.startswith("[repeat_setup"):
                setup = float(line.split()[1])
        if len(ts) != passes:
            raise RuntimeError("reference run printed %d of %d pass timers" % (len(ts), passes))
        return ts, setup, "reference", "the reference's LaplaceFMM hot block (P2M..P2P) repeated after one set-up"
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import rtfmm_oracle as orc
    ts = []
    for _ in range(passes):
        F = orc.FMM(x, q, W["P"], W["ncrit"], W["images"], W["cycle"], center=(0.5, 0.5, 0.5), divide_4pi=1)
        t0 = time.perf_counter()
        F.solve()
        ts.append(time.perf_counter() - t0)
    return ts, None, "port", "numpy oracle pass (single process)"


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    n = args.ref_n
    ts, setup, kind, note = reference_passes(n, threads, args.warmup + args.steps)
    timed = ts[args.warmup:]
    value = n / float(np.mean(timed))
    # the published runs used 8 threads (3dpp/exp/test_i.sh:17): two passes
    # at that setting beside the all-core figure
    th8 = None
    if threads != 8 and kind == "reference":
        t8, _, _, _ = reference_passes(n, 8, 2)
        th8 = {"value": n / t8[-1], "unit": "particles/s", "threads": 8}
    W = WORKLOAD
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "particles/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * n / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic: uniform [0,1)^3, q~U[-1,1] net zero, seed 2",
            "config": {"workload": "periodic KIFMM evaluation pass N=%d P=8 ncrit=256 images=3" % n,
                       "N": n, "P": W["P"], "ncrit": W["ncrit"], "images": W["images"], "cycle": W["cycle"],
                       "reference_setup_s": setup, "pass_s": timed, "cpu_model": cpu_model(),
                       "threads_8": th8},
            "cpu_baseline": {"value": value, "unit": "particles/s", "cores": threads, "kind": kind,
                             "sample": "N=%d bodies%s, %d timed passes after %d warm-up; %s"
                                       % (n, " (the full workload)" if n == W["N"] else "", args.steps,
                                          args.warmup, note)},
            "e2e": {"value": value, "unit": "particles/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
# our arm
# ----------------------------------------------------------------------------
def pass_error(phi, grad, phi_ref, grad_ref):
    """compare's relative L2 norms (3dpp/src/body.cpp:131-175): gradient, and
    potential with the mean difference removed (periodic potentials carry an
    implementation-dependent near-constant shift).  The larger of the two is
    the form's error."""
    d = phi - phi_ref
    eg = float(np.linalg.norm(grad - grad_ref) / np.linalg.norm(grad_ref))
    ep = float(np.linalg.norm(d - d.mean()) / np.linalg.norm(phi_ref - phi_ref.mean()))
    return eg, ep


def equal_error(pkg, mk, x, q, ref, w_dev, dq_dev, dx_dev, adj_ref, bound, steps):
    """Both forms timed over a grid of expansion orders and leaf sizes, each
    setting's error taken against the FP64 form at the workload's own settings
    (P=8, ncrit=256: the reference's FP64 FMM on the same input, to 1e-13).
    Every setting is timed on the pass and on forward + adjoint (the adjoint
    reusing the forward gradient), and its adjoint's dL/dx and dL/dq are
    compared with the FP64 adjoint at the workload's settings.  For each error
    bound the fastest FP64 and FP32-mixed settings within it are compared:
    on the pass by the pass's error, on forward + adjoint by the larger of the
    pass's and the adjoint's errors."""
    import torch
    phi_ref, grad_ref = ref
    grid = []
    for prec in (pkg.FP64, pkg.FP32_MIXED):
        for P in (5, 6, 7, 8):
            for ncrit in (64, 256, 512):
                f = pkg.LaplaceFMM(x, q, mk(prec, P=P, ncrit=ncrit))
                f.setup()
                f.upload()
                for _ in range(3):
                    f.evaluate_device()
                ms = []
                for _ in range(steps):
                    f.flush_l2()
                    ms.append(f.evaluate_device())
                eg, ep = pass_error(*f.download(), phi_ref, grad_ref)
                fa = []
                for k in range(2 + steps):
                    f.flush_l2()
                    t = f.evaluate_device() + f.adjoint_device(w_dev.data_ptr(), dq_dev.data_ptr(),
                                                                dx_dev.data_ptr())
                    if k >= 2:
                        fa.append(t)
                ax, aq = pass_error(dq_dev.cpu().numpy(), dx_dev.cpu().numpy(), adj_ref[0], adj_ref[1])
                grid.append({"form": "fp64" if prec == pkg.FP64 else "mixed", "P": P, "ncrit": ncrit,
                             "ms": float(np.median(ms)), "err_grad": eg, "err_phi_mr": ep, "err": max(eg, ep),
                             "fwd_adj_ms": float(np.median(fa)), "adj_err_dLdx": ax, "adj_err_dLdq_mr": aq,
                             "fwd_adj_err": max(eg, ep, ax, aq)})
                f.close()

    def fastest(form, key_err, key_ms, e):
        ok = [g for g in grid if g["form"] == form and g[key_err] <= e]
        return min(ok, key=lambda g: g[key_ms]) if ok else None

    out = []
    for name, e in bound:
        row = {"bound": name, "err_bound": e}
        a, b = fastest("fp64", "err", "ms", e), fastest("mixed", "err", "ms", e)
        row.update({"pass_fp64": a, "pass_mixed": b, "pass_speedup": a["ms"] / b["ms"] if a and b else None})
        a, b = fastest("fp64", "fwd_adj_err", "fwd_adj_ms", e), fastest("mixed", "fwd_adj_err", "fwd_adj_ms", e)
        row.update({"fwd_adj_fp64": a, "fwd_adj_mixed": b,
                    "fwd_adj_speedup": a["fwd_adj_ms"] / b["fwd_adj_ms"] if a and b else None})
        out.append(row)
    torch.cuda.synchronize()
    return {"reference_form": "FP64 P=8 ncrit=256, the workload's settings", "grid": grid, "targets": out}


def max_over_ranks(vals, world, device):
    """The timings of every rank replaced by their maximum over ranks (one
    all-reduce on the process group); unchanged on one rank.  Every rank
    calls it at the same point."""
    if world <= 1:
        return [float(v) for v in vals]
    import torch
    import torch.distributed as dist
    v = torch.tensor([float(x) for x in vals], dtype=torch.float64, device=device)
    dist.all_reduce(v, op=dist.ReduceOp.MAX)
    return v.tolist()


def replica_value(n_per_rank, world, ms_max):
    """Whole-job throughput of N independent replicas: all ranks' bodies over
    the slowest rank's pass time."""
    return world * n_per_rank / (ms_max * 1e-3)


def run_ours(args):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    pkg = load_pkg()
    W = WORKLOAD
    n = args.n
    x, q = make_bodies(n, W["seed"])
    mk = lambda prec, stages=pkg.STAGE_ALL, P=W["P"], ncrit=W["ncrit"]: pkg.Argument(
        P=P, ncrit=ncrit, images=W["images"], cycle=W["cycle"], x=(0.5, 0.5, 0.5),
        dipole_correction=0, divide_4pi=1, precision=prec, stages=stages, device=local)
    t0 = time.perf_counter()
    fm = pkg.LaplaceFMM(x, q, mk(pkg.FP32_MIXED))
    fm.setup()
    setup_s = time.perf_counter() - t0
    fm.upload()
    f64 = pkg.LaplaceFMM(x, q, mk(pkg.FP64))
    f64.setup()
    f64.upload()
    info = fm.info()
    setup_phases = fm.setup_times()  # first setup on the handle: operators included

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(f, steps, warmup):
        for _ in range(warmup):
            f.evaluate_device()
        barrier()
        ms = []
        for _ in range(steps):
            f.flush_l2()
            ms.append(f.evaluate_device())
        barrier()
        return ms

    with ClockSampler(local) as clk:
        ms_mixed = timed(fm, args.steps, args.warmup)
    launches = fm.launch_count() * args.steps
    ms64 = timed(f64, args.steps, max(1, args.warmup // 2))
    phi_m, grad_m = fm.download()
    phi_d, grad_d = f64.download()
    err = pkg.compare(phi_m, grad_m, q, phi_d, grad_d, q)
    dphi = phi_m - phi_d
    err_mr = float(np.linalg.norm(dphi - dphi.mean()) / np.linalg.norm(phi_d - phi_d.mean()))
    # both forms against the converged Ewald sum (FP64, GPU) on 1024 sampled
    # bodies; the FMM outputs carry 1/(4 pi) and no dipole correction, the
    # Ewald sum neither: grad_Ewald = 4 pi grad - (4 pi / 3 L^3) sum q x
    ts = np.random.default_rng(7).choice(n, 1024, replace=False)
    _, egrad = pkg.ewald_sampled(x, q, W["cycle"], ts, ksize=11, device=local)
    corr = 4 * math.pi / (3 * W["cycle"] ** 3) * (q @ x)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    err_ewald = {"grad_l2_fp64": rel(4 * math.pi * grad_d[ts] - corr, egrad),
                 "grad_l2_mixed": rel(4 * math.pi * grad_m[ts] - corr, egrad), "sampled_bodies": 1024,
                 "ksize": 11}

    # per-stage times of the overlapped pass: the same launches issued
    # directly with stage events instead of replayed as a CUDA graph
    ft = pkg.LaplaceFMM(x, q, mk(pkg.FP32_MIXED, pkg.STAGE_ALL | pkg.STAGE_TIMED))
    ft.setup()
    ft.upload()
    ms_direct = timed(ft, max(3, args.steps // 2), 2)
    st_mixed = ft.stage_times()
    ft.close()

    # per-stage times with the stages serialised (diagnostic only)
    fs = pkg.LaplaceFMM(x, q, mk(pkg.FP32_MIXED, pkg.STAGE_ALL | pkg.STAGE_SERIAL))
    fs.setup()
    fs.upload()
    for _ in range(2):
        fs.evaluate_device()
    ser = []
    for _ in range(max(3, args.steps // 2)):
        fs.flush_l2()
        fs.evaluate_device()
        ser.append(fs.stage_times())
    stage_serial = {k: float(np.mean([s[k] for s in ser])) for k in ser[0]}
    fs.close()

    # a new body set from device memory: GPU octree, P2P walk and P2P tables
    # (rtfmm_b200_setup_device, operators cached on the handle), then the pass
    xd = torch.from_numpy(x).cuda(local)
    qd = torch.from_numpy(q).cuda(local)
    fdv = pkg.LaplaceFMM(x, q, mk(pkg.FP32_MIXED))
    fdv.setup_device(xd.data_ptr(), qd.data_ptr(), n)  # operators built here
    sd_ms, sp_ms = [], []
    for _ in range(4):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fdv.setup_device(xd.data_ptr(), qd.data_ptr(), n)
        t1 = time.perf_counter()
        fdv.evaluate_device()
        t2 = time.perf_counter()
        sd_ms.append(1e3 * (t1 - t0))
        sp_ms.append(1e3 * (t2 - t0))
    device_setup = {"setup_ms": float(np.median(sd_ms)), "setup_plus_pass_ms": float(np.median(sp_ms)),
                    "phases_s": fdv.setup_times()}
    fdv.close()
    del xd, qd

    # end to end through the C ABI: pinned host charges in, pinned outputs back
    qh = torch.from_numpy(q.copy()).pin_memory()
    ph = torch.empty(n, dtype=torch.float64).pin_memory()
    gh = torch.empty((n, 3), dtype=torch.float64).pin_memory()
    qn, pn, gn = qh.numpy(), ph.numpy(), gh.numpy()
    lib = pkg.lib()
    import ctypes
    dp = ctypes.POINTER(ctypes.c_double)
    call = lambda: lib.rtfmm_b200_evaluate(fm._h, qn.ctypes.data_as(dp), pn.ctypes.data_as(dp),
                                           gn.ctypes.data_as(dp))
    for _ in range(args.warmup):
        assert call() == 0
    barrier()
    e2e = []
    for _ in range(args.steps):
        fm.flush_l2()
        t0 = time.perf_counter()
        assert call() == 0
        e2e.append(time.perf_counter() - t0)
    barrier()

    # forward + adjoint, both precisions: the comparison of the mixed and
    # FP64 forms on the full step.  Device-resident (CUDA events on the
    # solver's stream; the adjoint reuses the forward pass's gradient), and
    # through the host-buffer C ABI (wall clock) beside it.
    wts = np.random.default_rng(4).standard_normal(n)
    w_dev = torch.from_numpy(wts).cuda()
    dq_dev = torch.empty(n, dtype=torch.float64, device="cuda")
    dx_dev = torch.empty((n, 3), dtype=torch.float64, device="cuda")

    def fwd_adj_dev(f):
        f.flush_l2()
        t = f.evaluate_device()
        return t + f.adjoint_device(w_dev.data_ptr(), dq_dev.data_ptr(), dx_dev.data_ptr())

    def fwd_adj_host(f):
        t0 = time.perf_counter()
        f.evaluate(q)
        f.adjoint(wts)
        return 1000 * (time.perf_counter() - t0)

    for f in (fm, f64):
        fwd_adj_dev(f)
        fwd_adj_host(f)
    fa_m = float(np.mean([fwd_adj_dev(fm) for _ in range(max(3, args.steps // 2))]))
    fa_d = float(np.mean([fwd_adj_dev(f64) for _ in range(max(3, args.steps // 2))]))
    fh_m = float(np.mean([fwd_adj_host(fm) for _ in range(2)]))
    fh_d = float(np.mean([fwd_adj_host(f64) for _ in range(2)]))
    # accuracy of the mixed adjoint against the FP64 one
    fm.evaluate_device()
    fm.adjoint_device(w_dev.data_ptr(), dq_dev.data_ptr(), dx_dev.data_ptr())
    dq_m, dx_m = dq_dev.cpu().numpy(), dx_dev.cpu().numpy()
    f64.evaluate_device()
    f64.adjoint_device(w_dev.data_ptr(), dq_dev.data_ptr(), dx_dev.data_ptr())
    dq_d, dx_d = dq_dev.cpu().numpy(), dx_dev.cpu().numpy()
    ddq = dq_m - dq_d
    adj_err = {"dLdq_l2": float(np.linalg.norm(ddq) / np.linalg.norm(dq_d)),
               "dLdq_l2_mean_removed": float(np.linalg.norm(ddq - ddq.mean()) / np.linalg.norm(dq_d - dq_d.mean())),
               "dLdx_l2": float(np.linalg.norm(dx_m - dx_d) / np.linalg.norm(dx_d))}

    t_m = float(np.mean(ms_mixed))
    t_d = float(np.mean(ms64))
    t_e = float(np.mean(e2e))
    # the FP32-mixed form against the FP64 form at equal error (one GPU)
    eq_err = None
    if world == 1 and not args.no_equal_error:
        eq_err = equal_error(pkg, mk, x, q, (phi_d, grad_d), w_dev, dq_dev, dx_dev, (dq_d, dx_d),
                             [("1e-5 accuracy bound", 1e-5),
                              ("mixed form's own error at P=8 ncrit=256", max(err["l2f"], err_mr))],
                             max(3, args.steps // 2))
    t_m, t_d, t_e = max_over_ranks([t_m, t_d, t_e], world, "cuda")
    if rank != 0:
        dist.destroy_process_group()
        return
    clocks = clk.summary()
    # roofline of the dominant kernel, from the serialised stage times
    hbm, hbm_kind = measured_peaks()
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    P = W["P"]
    N = 2 * P - 1
    Nf = N * N * P
    # the Hadamard's algorithmic work: a complex 8x8 block (64 complex MACs =
    # 512 flop) per filled (target parent, direction) pair and frequency;
    # bytes: source spectra read once, target spectra read and written (8
    # complex FP32 slots each), the 26 x 64 kernel spectra once
    had_flop = 8.0 * 64 * Nf * info["m2l8_pairs"]
    had_bytes = Nf * 8 * 8 * (info["m2l8_sources"] + 2 * info["m2l8_targets"]) + 26 * 64 * Nf * 8
    kern = {
        "p2p32": {"bound": "fp32", "work": 20.0 * info["p2p_pairs"], "ms": stage_serial["P2P"],
                  "peak": fp32_peak, "unit": "TFLOP/s",
                  "peak_kind": "nominal 148 SM x 128 FMA/clk x 2 at the sampled SM clock"},
        "m2l_hadamard8": {"bound": "fp32", "work": had_flop, "ms": stage_serial["M2L_hadamard"],
                          "peak": fp32_peak, "unit": "TFLOP/s",
                          "peak_kind": "nominal FP32 at the sampled SM clock; against the measured HBM peak "
                                       "it moves %.0f MB" % (had_bytes / 1e6)},
    }
    for k, d in kern.items():
        scale = 1e12 if d["unit"] == "TFLOP/s" else 1e9
        d["achieved"] = d["work"] / (d["ms"] * 1e-3) / scale if d["ms"] > 0 else None
        d["frac"] = d["achieved"] / d["peak"] if d["achieved"] else None
    top = max(kern, key=lambda k: kern[k]["ms"])
    K = kern[top]
    roofline = {"kernel": top, "bound": K["bound"], "achieved": K["achieved"], "peak": K["peak"],
                "unit": K["unit"], "frac": K["frac"], "peak_kind": K["peak_kind"],
                "traffic": read_traffic(top),
                "work_per_launch": K["work"], "launch_ms": K["ms"],
                "others": {k: {"achieved": d["achieved"], "peak": d["peak"], "unit": d["unit"],
                               "frac": d["frac"], "launch_ms": d["ms"]} for k, d in kern.items() if k != top}}
    pass_roof = pass_roofline(info, n, Nf, had_flop, had_bytes, fp32_peak, sm_mhz, hbm, hbm_kind, t_m)
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            ncores = os.cpu_count() or 1
            ts, setup, kind, note = reference_passes(args.ref_n, ncores, 2)
            cpu = {"value": args.ref_n / ts[-1], "unit": "particles/s", "cores": ncores, "kind": kind,
                   "sample": "N=%d bodies of the workload (P=8 ncrit=256 images=3), the second of two passes "
                             "after one set-up (%.1f s); %s" % (args.ref_n, setup or 0.0, note),
                   "cpu_model": cpu_model()}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "particles/s", "cores": 0, "kind": "none", "sample": "failed: %s" % e}
    line = {
        "metric": METRIC, "value": replica_value(n, world, t_m), "unit": "particles/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_m, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32-mixed",
        "data": "synthetic: uniform [0,1)^3, q~U[-1,1] net zero, seed 2",
        "config": {"workload": "periodic KIFMM evaluation pass N=%d P=8 ncrit=256 images=3" % n,
                   "N": n, "P": P, "ncrit": W["ncrit"], "images": W["images"], "cycle": W["cycle"],
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "256 MB flush between timed steps",
                   "setup_s": setup_s, "setup_phases_s": setup_phases,
                   "nleaf": info["nleaf"], "ncell": info["ncell"],
                   "p2p_pairs": info["p2p_pairs"],
                   "fp64_ms_per_step": t_d, "fp64_value": replica_value(n, world, t_d),
                   "mixed_speedup_vs_fp64": t_d / t_m,
                   "mixed_err_vs_fp64": {"l2p": err["l2p"], "l2f": err["l2f"], "l2p_mean_removed": err_mr},
                   "err_vs_ewald_sampled": err_ewald,
                   "device_setup": device_setup,
                   "fwd_adj_ms_mixed": fa_m, "fwd_adj_ms_fp64": fa_d,
                   "fwd_adj_mixed_speedup_vs_fp64": fa_d / fa_m,
                   "fwd_adj_mixed_err_vs_fp64": adj_err,
                   "equal_error": eq_err,
                   "fwd_adj_host_ms_mixed": fh_m, "fwd_adj_host_ms_fp64": fh_d,
                   "pass_launch": "CUDA graph replay",
                   "ms_per_step_direct_launches": float(np.median(ms_direct)),
                   "stage_ms_overlapped": st_mixed, "stage_ms_serial": stage_serial},
        "roofline": roofline,
        "pass_roofline": pass_roof,
        "cpu_baseline": cpu,
        "e2e": {"value": world * n / t_e, "unit": "particles/s", "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 8 * n + 24 * n, "ms_per_step": 1000 * t_e},
        "gpu_launches": launches,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


# ----------------------------------------------------------------------------
# the other large configurations (one JSON line each; the headline is C2)
# ----------------------------------------------------------------------------
def config_bodies(name):
    """C3: 2^22 bodies in 64 Gaussian blobs (centres U[0,1)^3, sigma 0.02,
    wrapped mod 1), charges +-1 balanced to net zero, seed 3.  C5: the 200^3
    rock-salt lattice of spacing 1/200, each site jittered by U(+-0.1
    spacing) per axis, charges (-1)^(i+j+k), seed 5."""
    if name == "c3":
        rng = np.random.default_rng(3)
        n, nb = 1 << 22, 64
        c = rng.random((nb, 3))
        x = np.mod(c[rng.integers(0, nb, n)] + 0.02 * rng.standard_normal((n, 3)), 1.0)
        q = np.where(rng.random(n) < 0.5, -1.0, 1.0)
        return x, q - q.mean(), dict(P=10, ncrit=128, images=3)
    m = 200
    a = 1.0 / m
    g = (np.arange(m) + 0.5) * a
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    x = np.mod(x + np.random.default_rng(5).uniform(-0.1 * a, 0.1 * a, x.shape), 1.0)
    i, j, k = np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij")
    q = np.where((i + j + k).ravel() % 2 == 0, 1.0, -1.0)
    return x, q, dict(P=10, ncrit=256, images=4)


def run_shard(args):
    """The pass sharded over the ranks (rtfmm_b200_shard): every rank sets up
    the headline workload, computes its share of the bodies, and the ranks
    exchange once per pass (an NCCL all-reduce of the leaf q_equiv rows, 43 MB
    at N=2^20, P=8).  Total work is fixed: strong scaling.  A step is the
    upward phase, the all-reduce and the downward phase, bracketed by device
    synchronisations on every rank and timed with CUDA events on the current
    stream (the library's phases synchronise their own streams); the max over
    ranks is reported."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    pkg = load_pkg()
    W = WORKLOAD
    x, q = make_bodies(args.n, W["seed"])
    n = len(q)
    a = pkg.Argument(P=W["P"], ncrit=W["ncrit"], images=W["images"], cycle=W["cycle"], x=(0.5, 0.5, 0.5),
                     dipole_correction=0, divide_4pi=1, precision=pkg.FP32_MIXED, device=local)
    f = pkg.LaplaceFMM(x, q, a)
    f.shard(rank, world)
    f.setup()
    f.upload()
    nb, nx = f.shard_sizes()
    xbuf = torch.empty(nx, dtype=torch.float64, device="cuda")
    phi = torch.empty(n, dtype=torch.float64, device="cuda")
    grad = torch.empty((n, 3), dtype=torch.float64, device="cuda")

    def step():
        f.shard_upward(xbuf.data_ptr())
        if world > 1:
            dist.all_reduce(xbuf)
            torch.cuda.synchronize()
        f.shard_downward(xbuf.data_ptr(), phi.data_ptr(), grad.data_ptr())

    for _ in range(args.warmup):
        step()
    ms = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            f.flush_l2()
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            e0.record()
            step()
            torch.cuda.synchronize()
            e1.record()
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
    t = max_over_ranks([float(np.mean(ms))], world, "cuda")[0]
    f.close()
    if rank == 0:
        line = {"metric": METRIC, "value": n / (t * 1e-3), "unit": "particles/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": t, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32-mixed",
                "data": "synthetic: uniform [0,1)^3, q~U[-1,1] net zero, seed 2",
                "config": {"workload": "periodic KIFMM evaluation pass N=%d P=8 ncrit=256 images=3, sharded" % n,
                           "N": n, "parallelism": "shard%d" % world, "bodies_rank0": nb,
                           "exchange_bytes": 8 * nx, "l2": "256 MB flush between timed steps"},
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


CONFIG_DATA = {
    "c3": "synthetic: 2^22 bodies in 64 Gaussian blobs (sigma 0.02, wrapped), q=+-1 net zero, seed 3",
    "c5": "synthetic: 200^3 rock-salt lattice jittered by U(+-0.1 spacing), q=(-1)^(i+j+k), seed 5",
}


def run_config(args):
    """One configuration other than the headline: both forms' pass and
    forward + adjoint times (device-resident, CUDA events, L2 flushed between
    steps) and the mixed form's errors against the FP64 form."""
    import torch
    torch.cuda.set_device(0)
    pkg = load_pkg()
    x, q, c = config_bodies(args.config)
    n = len(q)
    mk = lambda prec: pkg.Argument(P=c["P"], ncrit=c["ncrit"], images=c["images"], cycle=1.0, x=(0.5, 0.5, 0.5),
                                   dipole_correction=0, divide_4pi=1, precision=prec, device=0)
    w_dev = torch.from_numpy(np.random.default_rng(4).standard_normal(n)).cuda()
    dq_dev = torch.empty(n, dtype=torch.float64, device="cuda")
    dx_dev = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    res = {}
    with ClockSampler(0) as clk:
        for prec in (pkg.FP64, pkg.FP32_MIXED):
            f = pkg.LaplaceFMM(x, q, mk(prec))
            t0 = time.perf_counter()
            f.setup()
            f.upload()
            setup_s = time.perf_counter() - t0
            for _ in range(args.warmup):
                f.evaluate_device()
            ms = []
            for _ in range(args.steps):
                f.flush_l2()
                ms.append(f.evaluate_device())
            phi, grad = f.download()
            fa = []
            for k in range(1 + max(2, args.steps // 2)):
                f.flush_l2()
                t = f.evaluate_device() + f.adjoint_device(w_dev.data_ptr(), dq_dev.data_ptr(), dx_dev.data_ptr())
                if k:
                    fa.append(t)
            res[prec] = dict(ms=float(np.median(ms)), fwd_adj_ms=float(np.median(fa)), phi=phi, grad=grad,
                             dq=dq_dev.cpu().numpy(), dx=dx_dev.cpu().numpy(), setup_s=setup_s, info=f.info())
            f.close()
    d, m = res[pkg.FP64], res[pkg.FP32_MIXED]
    eg, ep = pass_error(m["phi"], m["grad"], d["phi"], d["grad"])
    ax, aq = pass_error(m["dq"], m["dx"], d["dq"], d["dx"])
    line = {"metric": METRIC.replace("N=1M P=8", "%s N=%d P=%d" % (args.config.upper(), n, c["P"])),
            "value": n / (m["ms"] * 1e-3), "unit": "particles/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": m["ms"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32-mixed", "data": CONFIG_DATA[args.config],
            "config": {"workload": "periodic KIFMM evaluation pass %s" % args.config.upper(), "N": n, **c,
                       "l2": "256 MB flush between timed steps", "nleaf": m["info"]["nleaf"],
                       "ncell": m["info"]["ncell"], "p2p_pairs": m["info"]["p2p_pairs"],
                       "close_pairs": m["info"]["close_pairs"],
                       "fp64_ms_per_step": d["ms"], "mixed_speedup_vs_fp64": d["ms"] / m["ms"],
                       "mixed_err_vs_fp64": {"l2f": eg, "l2p_mean_removed": ep},
                       "fwd_adj_ms_mixed": m["fwd_adj_ms"], "fwd_adj_ms_fp64": d["fwd_adj_ms"],
                       "fwd_adj_mixed_speedup_vs_fp64": d["fwd_adj_ms"] / m["fwd_adj_ms"],
                       "fwd_adj_mixed_err_vs_fp64": {"dLdx_l2": ax, "dLdq_l2_mean_removed": aq},
                       "setup_s": {"fp64": d["setup_s"], "mixed": m["setup_s"]}},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=WORKLOAD["N"])
    ap.add_argument("--ref-n", type=int, default=WORKLOAD["N"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-equal-error", action="store_true")
    ap.add_argument("--shard", action="store_true",
                    help="the pass sharded over the ranks (one all-reduce per pass) instead of replicas")
    ap.add_argument("--config", default="c2", choices=["c2", "c3", "c5"],
                    help="c2: the headline workload (default); c3, c5: the clustered and lattice configurations")
    args = ap.parse_args()
    if args.config != "c2":
        run_config(args)
    elif args.shard and args.impl == "ours":
        run_shard(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
