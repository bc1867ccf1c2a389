"""The multi-GPU path of bench.py is replicas only (the pass does not shard
in this build): each rank runs its own pass and rank 0 reports all ranks'
bodies over the slowest rank's time.  Checked here with two gloo ranks on
CPU: the max-over-ranks reduction and the aggregate value."""
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
