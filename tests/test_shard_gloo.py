"""The pass sharded over ranks, on CPU: the partition rule and the one
exchange step of rtfmm_b200_shard, run by the numpy oracle in two gloo
processes (torch.distributed all-reduce of the leaf q_equiv rows).

Rank r computes the leaves whose first body (tree order) lies in
[r n / R, (r + 1) n / R) and the cells above them: P2M of its leaves, then
the exchange (the leaf rows summed over the ranks; each rank contributes its
own rows and zeros elsewhere), then M2M on the whole tree, M2L and L2L of
its cells, L2P and P2P of its leaves.  Every body is computed by exactly one
rank, and its outputs equal the single-rank pass's.  The GPU library's
sharded pass (same rule, same phases) is checked against its unsharded pass
in tests/test_gpu_shard.py.
"""
import os

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASE = dict(n=2500, P=4, ncrit=32, images=2, seed=31)


def bodies():
    rng = np.random.default_rng(CASE["seed"])
    x = rng.random((CASE["n"], 3))
    q = rng.random(CASE["n"]) * 2 - 1
    return x, q - q.mean()


def make_fmm(orc):
    x, q = bodies()
    return orc.FMM(x, q, CASE["P"], CASE["ncrit"], CASE["images"], 1.0, center=(0.5, 0.5, 0.5), divide_4pi=1)


def _rank(rank, world, port, out):
    import datetime
    import sys

    import torch
    import torch.distributed as dist
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import rtfmm_oracle as orc
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        def allreduce(buf):
            t = torch.from_numpy(buf)  # shares the array's memory
            dist.all_reduce(t, op=dist.ReduceOp.SUM)

        out[rank] = make_fmm(orc).solve_sharded(rank, world, allreduce)
    finally:
        dist.destroy_process_group()


def check(parts, oracle):
    phi, grad = make_fmm(oracle).solve()
    seen = np.zeros(len(phi), int)
    for p, g, m in parts:
        seen += m
        assert np.abs(p[m] - phi[m]).max() <= 1e-13 * np.abs(phi).max()
        assert np.abs(g[m] - grad[m]).max() <= 1e-13 * np.abs(grad).max()
    assert (seen == 1).all()  # every body computed by exactly one rank


def test_sharded_pass_two_gloo_ranks(oracle):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = 29700 + os.getpid() % 1000
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        check([out[0], out[1]], oracle)


def test_sharded_pass_three_ranks_in_sequence(oracle):
    """Three ranks, run one after the other with the exchange done by hand:
    each contributes its rows, then every rank continues from the sum."""
    fmms = [make_fmm(oracle) for _ in range(3)]
    bufs = {}

    # phase 1 of every rank, then the sum, then phase 2: solve_sharded calls
    # the exchange between them, so record each rank's rows first
    def record(r):
        def allreduce(buf):
            bufs[r] = buf.copy()
            raise StopIteration
        return allreduce

    for r in range(3):
        try:
            fmms[r].solve_sharded(r, 3, record(r))
        except StopIteration:
            pass
    total = sum(bufs.values())
    parts = []
    for r in range(3):
        f = make_fmm(oracle)

        def allreduce(buf):
            buf[...] = total

        parts.append(f.solve_sharded(r, 3, allreduce))
    check(parts, oracle)
    # the ranks' shares of the bodies are balanced to within one leaf
    counts = [int(p[2].sum()) for p in parts]
    assert max(counts) - min(counts) <= 2 * CASE["ncrit"]
