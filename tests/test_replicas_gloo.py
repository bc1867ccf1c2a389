"""bench.py's multi-GPU bookkeeping.  By default each rank runs its own
pass (replicas; --shard splits one pass instead) and rank 0 reports all
ranks' bodies over the slowest rank's time: the max-over-ranks reduction and
the aggregate value, with two gloo ranks on CPU.  Also the whole-pass
roofline helper, on the headline workload's counts."""
import importlib.util
import os

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("rtfmm_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench = load_bench()
        # rank r took (r + 1) ms on its pass, 10 - r on the FP64 pass
        t = bench.max_over_ranks([rank + 1.0, 10.0 - rank, 5.0], world, "cpu")
        out[rank] = (t, bench.replica_value(1000, world, t[0]))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = 29500 + os.getpid() % 1000
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        for r in range(2):
            t, value = out[r]
            assert t == [2.0, 10.0, 5.0]
            assert value == pytest.approx(2 * 1000 / 2.0e-3)


def test_single_rank_is_unchanged():
    bench = load_bench()
    assert bench.max_over_ranks([1.5, 2.5], 1, "cpu") == [1.5, 2.5]
    assert bench.replica_value(1 << 20, 1, 7.0) == pytest.approx((1 << 20) / 7.0e-3)


def test_pass_roofline_sums_stage_bounds():
    bench = load_bench()
    # counts of the headline workload (N = 2^20, P = 8, ncrit = 256)
    info = {"num_surf": 296, "nleaf": 18075, "ncell": 20660, "p2p_pairs": 5601309424, "m2l8_pairs": 40214,
            "m2l8_sources": 2633, "m2l8_targets": 2581}
    Nf = 15 * 15 * 8
    had_flop = 8.0 * 64 * Nf * info["m2l8_pairs"]
    had_bytes = Nf * 64 * (2633 + 2 * 2581) + 26 * 64 * Nf * 8
    r = bench.pass_roofline(info, 1 << 20, Nf, had_flop, had_bytes, 74.45, 1965.0, 6542.1, "measured", 6.7)
    st = r["stages_bound_ms"]
    assert set(st) == {"P2P", "P2M", "M2M", "M2L_up", "M2L_hadamard", "M2L_down", "L2L", "L2P"}
    # P2P is FP32-bound: 20 flop per pair at 74.45 TFLOP/s
    assert abs(st["P2P"] - 20.0 * 5601309424 / 74.45e12 * 1e3) < 1e-9
    # the spectra passes are bandwidth-bound
    assert abs(st["M2L_up"] - (8.0 * 296 * 8 + 8.0 * Nf * 8) * 2633 / 6542.1e9 * 1e3) < 1e-9
    assert abs(r["bound_ms"] - sum(st.values())) < 1e-9
    assert abs(r["frac"] - r["bound_ms"] / 6.7) < 1e-12 and 0.2 < r["frac"] < 1.0

