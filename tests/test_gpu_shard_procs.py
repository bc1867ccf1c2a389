"""The sharded pass as it runs in a job: two processes (torch.distributed,
gloo), each a rank with its own handle and CUDA context, the exchange an
all-reduce between them.  Both processes share the one GPU of this test
machine; their kernels never wait on one another (the exchange is between
launches, through host memory), so that is safe and is the same pass as two
GPUs.  Each rank's bodies equal the unsharded pass's bit for bit."""
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CASE = dict(n=40000, seed=61, P=6, ncrit=64, images=3)


def bodies():
    rng = np.random.default_rng(CASE["seed"])
    x = rng.random((CASE["n"], 3))
    q = rng.random(CASE["n"]) * 2 - 1
    return x, q - q.mean()


def _rank(rank, world, port, precision, out):
    import datetime
    import importlib.util
    import sys

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    pkg = bench.load_pkg()
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        x, q = bodies()
        n = len(q)
        a = pkg.Argument(P=CASE["P"], ncrit=CASE["ncrit"], images=CASE["images"], cycle=1.0,
                         x=(0.5, 0.5, 0.5), dipole_correction=0, divide_4pi=1, precision=precision)
        f = pkg.LaplaceFMM(x, q, a)
        f.shard(rank, world)
        f.setup()
        f.upload()
        _, nx = f.shard_sizes()
        xbuf = torch.empty(nx, dtype=torch.float64, device="cuda")
        phi = torch.empty(n, dtype=torch.float64, device="cuda")
        grad = torch.empty((n, 3), dtype=torch.float64, device="cuda")
        for _ in range(2):
            f.shard_upward(xbuf.data_ptr())
            host = xbuf.cpu()
            dist.all_reduce(host)  # gloo: the sum through host memory
            xbuf.copy_(host)
            torch.cuda.synchronize()
            f.shard_downward(xbuf.data_ptr(), phi.data_ptr(), grad.data_ptr())
        idx = f.shard_bodies()
        out[rank] = (idx, phi.cpu().numpy()[idx], grad.cpu().numpy()[idx])
        f.close()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("precision", [0, 1])
def test_two_processes_equal_unsharded(pkg, precision):
    import torch
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = 29900 + os.getpid() % 50 + 50 * precision
        procs = [ctx.Process(target=_rank, args=(r, 2, port, precision, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        parts = [out[0], out[1]]
    x, q = bodies()
    a = pkg.Argument(P=CASE["P"], ncrit=CASE["ncrit"], images=CASE["images"], cycle=1.0, x=(0.5, 0.5, 0.5),
                     dipole_correction=0, divide_4pi=1, precision=precision)
    f = pkg.LaplaceFMM(x, q, a)
    f.setup()
    f.upload()
    f.evaluate_device()
    phi, grad = f.download()
    f.close()
    torch.cuda.synchronize()
    seen = np.zeros(len(q), int)
    for idx, p, g in parts:
        seen[idx] += 1
        assert np.array_equal(p, phi[idx]) and np.array_equal(g, grad[idx])
    assert (seen == 1).all()
