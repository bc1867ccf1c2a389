"""The pass sharded over ranks on the GPU (rtfmm_b200_shard): R handles, one
per rank share, run in turn on one GPU with the exchange (the sum of the
ranks' leaf q_equiv rows) done in between.  The ranks never wait on one
another inside a kernel, so running them in sequence is the same pass as
running them on R GPUs.  Each body is computed by exactly one rank and its
outputs equal the unsharded pass's bit for bit; both precisions, free space
and periodic."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def uniform01(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 3))
    q = rng.random(n) * 2 - 1
    return x, q - q.mean()


def args(pkg, precision, images, P=6, ncrit=64):
    return pkg.Argument(P=P, ncrit=ncrit, images=images, cycle=1.0, x=(0.5, 0.5, 0.5), dipole_correction=0,
                        divide_4pi=1, precision=precision)


def unsharded(pkg, x, q, a):
    import torch
    n = len(q)
    f = pkg.LaplaceFMM(x, q, a)
    f.setup()
    f.upload()
    phi = torch.empty(n, dtype=torch.float64, device="cuda")
    grad = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    f.forward_device(0, phi.data_ptr(), grad.data_ptr())
    f.close()
    return phi.cpu().numpy(), grad.cpu().numpy()


def sharded(pkg, x, q, a, R, passes=1):
    import torch
    n = len(q)
    hs = []
    for r in range(R):
        f = pkg.LaplaceFMM(x, q, a)
        f.shard(r, R)
        f.setup()
        f.upload()
        hs.append(f)
    nx = hs[0].shard_sizes()[1]
    outs = []
    for _ in range(passes):
        bufs = [torch.full((nx,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(R)]
        for f, b in zip(hs, bufs):
            f.shard_upward(b.data_ptr())
        total = torch.stack(bufs).sum(0)
        outs = []
        for f in hs:
            phi = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
            grad = torch.full((n, 3), float("nan"), dtype=torch.float64, device="cuda")
            assert f.shard_downward(total.data_ptr(), phi.data_ptr(), grad.data_ptr()) > 0
            outs.append((f.shard_bodies(), phi.cpu().numpy(), grad.cpu().numpy()))
    for f in hs:
        f.close()
    return outs


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("images,R", [(3, 3), (0, 2), (2, 1)])
def test_sharded_equals_unsharded(pkg, precision, images, R):
    x, q = uniform01(20000, 40 + R)
    a = args(pkg, precision, images)
    phi, grad = unsharded(pkg, x, q, a)
    seen = np.zeros(len(q), int)
    for idx, p, g in sharded(pkg, x, q, a, R, passes=2):
        seen[idx] += 1
        assert np.array_equal(p[idx], phi[idx])
        assert np.array_equal(g[idx], grad[idx])
    assert (seen == 1).all()


def test_sharded_handle_refuses_whole_pass_calls(pkg):
    x, q = uniform01(3000, 50)
    f = pkg.LaplaceFMM(x, q, args(pkg, 0, 2))
    f.shard(1, 2)
    f.setup()
    f.upload()
    with pytest.raises(pkg.RtfmmError) as e:
        f.evaluate_device()
    assert e.value.code == 4  # RTFMM_ESTATE
    with pytest.raises(pkg.RtfmmError) as e:
        f.shard(2, 2)
    assert e.value.code == 1
    # back to the whole pass at the next set-up
    f.shard(0, 1)
    f.setup()
    f.upload()
    assert f.evaluate_device() > 0
    f.close()
