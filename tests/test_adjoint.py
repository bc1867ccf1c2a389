"""The hand-written adjoint (rtfmm_b200_adjoint): for L = sum_i w_i phi_i it
returns dL/dq = K^T w and dL/dx, where K is the discretised FMM operator.

Checks: the transpose identity <w, K q> = <q, K^T w>; central finite
differences of dL/dx (h = 1e-4, FP64, 64 bodies away from cell faces); dL/dx for L = 1/2 sum q phi against q times the
reference's own gradient output; and the autograd harness.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def uniform01(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.random((n, 3))
    q = rng.random(n) * 2 - 1
    return x, q - q.mean()


def args(pkg, P, ncrit, images, precision=0):
    return pkg.Argument(P=P, ncrit=ncrit, images=images, cycle=1.0, x=(0.5, 0.5, 0.5), dipole_correction=0,
                        divide_4pi=1, precision=precision)


@pytest.mark.parametrize("images", [0, 3])
@pytest.mark.parametrize("precision,tol", [(0, 1e-11), (1, 2e-6)])
def test_transpose_identity(pkg, images, precision, tol):
    x, q = uniform01(3000, 5)
    rng = np.random.default_rng(6)
    w = rng.standard_normal(len(q))
    f = pkg.LaplaceFMM(x, q, args(pkg, 6, 32, images, precision))
    phi, _ = f.solve()
    dq, _ = f.adjoint(w)
    lhs = float(w @ phi)
    rhs = float(q @ dq)
    assert abs(lhs - rhs) / (np.linalg.norm(w) * np.linalg.norm(phi)) < tol, (lhs, rhs)
    # the FMM operator is nearly symmetric: K^T w is close to K w
    fw = pkg.LaplaceFMM(x, w, args(pkg, 6, 32, images, precision))
    phiw, _ = fw.solve()
    d = dq - phiw
    assert np.linalg.norm(d - d.mean()) / np.linalg.norm(phiw - phiw.mean()) < 1e-4


def away_from_faces(x, h, depth=8):
    """bodies at least 3h from every cell face down to `depth` levels."""
    ok = np.ones(len(x), bool)
    for d in range(1, depth + 1):
        s = x * (1 << d)
        ok &= np.all(np.abs(s - np.round(s)) > 3 * h * (1 << d), axis=1)
    return np.nonzero(ok)[0]


@pytest.mark.parametrize("images", [0, 2])
def test_position_gradient_by_finite_differences(pkg, images):
    x, q = uniform01(2000, 7)
    rng = np.random.default_rng(8)
    w = rng.standard_normal(len(q))
    a = args(pkg, 6, 32, images, 0)
    f = pkg.LaplaceFMM(x, q, a)
    f.solve()
    dq, dx = f.adjoint(w)
    h = 1e-4
    cand = away_from_faces(x, h)
    pick = rng.choice(cand, size=64, replace=False)

    def central(step):
        fd = np.zeros((64, 3))
        for r, i in enumerate(pick):
            for k in range(3):
                vals = []
                for sgn in (1, -1):
                    xp = x.copy()
                    xp[i, k] += sgn * step
                    g = pkg.LaplaceFMM(xp, q, a)
                    phi, _ = g.solve()
                    vals.append(float(w @ phi))
                    g.close()
                fd[r, k] = (vals[0] - vals[1]) / (2 * step)
        return fd

    fd_h = central(h)
    fd_h2 = central(h / 2)
    ref = dx[pick]
    # central differences at h = 1e-4 carry an O(h^2) truncation from close
    # body pairs; Richardson's extrapolation (4 f(h/2) - f(h))/3 removes it
    assert np.linalg.norm(fd_h - ref) / np.linalg.norm(ref) < 3e-5
    rich = (4 * fd_h2 - fd_h) / 3
    assert np.linalg.norm(rich - ref) / np.linalg.norm(ref) < 1e-7


def test_half_energy_gradient_matches_reference_force(pkg):
    """For L = 1/2 sum q phi, dL/dx_i = q_i (grad phi_i + grad psi_i)/2, which
    equals q_i times the reference's gradient output up to the FMM's
    asymmetry."""
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_c1_small.npz"))
    a = pkg.Argument(P=int(g["P"]), ncrit=int(g["ncrit"]), images=int(g["images"]), cycle=float(g["cycle"]),
                     dipole_correction=0, divide_4pi=int(g["divide_4pi"]))
    f = pkg.LaplaceFMM(g["x"], g["q"], a)
    f.solve()
    dq, dx = f.adjoint(0.5 * g["q"])
    ref = g["q"][:, None] * g["grad"]
    assert np.linalg.norm(dx - ref) / np.linalg.norm(ref) < 1e-4
    # with w = q/2 held fixed the adjoint gives K^T (q/2); the gradient of the
    # quadratic adds the explicit phi/2, and the sum is the potential up to
    # the same asymmetry (compared with the mean removed: periodic potentials)
    d = (dq + g["phi"] / 2) - g["phi"]
    assert np.linalg.norm(d - d.mean()) / np.linalg.norm(g["phi"] - g["phi"].mean()) < 1e-4


def test_autograd_harness(pkg):
    import torch
    from fmm_autograd import fmm_potential
    x, q = uniform01(1500, 9)
    a = args(pkg, 5, 32, 1, 0)
    xt = torch.tensor(x, requires_grad=True)
    qt = torch.tensor(q, requires_grad=True)
    w = torch.tensor(np.random.default_rng(10).standard_normal(len(q)))
    phi = fmm_potential(xt, qt, pkg, a)
    (phi * w).sum().backward()
    f = pkg.LaplaceFMM(x, q, a)
    f.solve()
    dq, dx = f.adjoint(w.numpy())
    assert np.allclose(qt.grad.numpy(), dq, rtol=0, atol=1e-12 * np.abs(dq).max())
    assert np.allclose(xt.grad.numpy(), dx, rtol=0, atol=1e-12 * np.abs(dx).max())


@pytest.mark.parametrize("precision,dipole", [(0, 0), (1, 0), (0, 1)])
def test_device_adjoint_matches_host_adjoint(pkg, precision, dipole):
    """rtfmm_b200_adjoint_device on device buffers gives the host adjoint's
    dL/dq and dL/dx: after a forward pass without the dipole correction it
    reuses that pass's gradient, otherwise (dipole on, or a second call) it
    recomputes it."""
    import torch
    x, q = uniform01(3000, 11)
    w = np.random.default_rng(12).standard_normal(len(q))
    a = pkg.Argument(P=6, ncrit=32, images=3, cycle=1.0, x=(0.5, 0.5, 0.5), dipole_correction=dipole,
                     divide_4pi=1, precision=precision)
    ref = pkg.LaplaceFMM(x, q, a)
    ref.setup()
    dq_ref, dx_ref = ref.adjoint(w)
    f = pkg.LaplaceFMM(x, q, a)
    f.setup()
    f.upload()
    f.evaluate_device()
    wt = torch.from_numpy(w).cuda()
    for call in range(2):
        dq = torch.full((len(q),), float("nan"), dtype=torch.float64, device="cuda")
        dx = torch.full((len(q), 3), float("nan"), dtype=torch.float64, device="cuda")
        ms = f.adjoint_device(wt.data_ptr(), dq.data_ptr(), dx.data_ptr())
        assert ms > 0
        dqn, dxn = dq.cpu().numpy(), dx.cpu().numpy()
        assert np.linalg.norm(dqn - dq_ref) <= 1e-12 * np.linalg.norm(dq_ref), call
        assert np.linalg.norm(dxn - dx_ref) <= 1e-12 * np.linalg.norm(dx_ref), call


@pytest.mark.parametrize("precision", [0, 1])
def test_forward_device_matches_host_solve(pkg, precision):
    """rtfmm_b200_forward_device with new charges on the device equals a host
    solve with those charges (same tree, same kernels)."""
    import torch
    x, q = uniform01(3000, 13)
    q2 = np.random.default_rng(14).standard_normal(len(q))
    q2 -= q2.mean()
    a = args(pkg, 6, 32, 3, precision)
    f = pkg.LaplaceFMM(x, q, a)
    f.setup()
    f.upload()
    qd = torch.from_numpy(q2).cuda()
    phi = torch.full((len(q),), float("nan"), dtype=torch.float64, device="cuda")
    grad = torch.full((len(q), 3), float("nan"), dtype=torch.float64, device="cuda")
    assert f.forward_device(qd.data_ptr(), phi.data_ptr(), grad.data_ptr()) > 0
    ref = pkg.LaplaceFMM(x, q2, a)
    rphi, rgrad = ref.solve()
    assert np.allclose(phi.cpu().numpy(), rphi, rtol=0, atol=1e-13 * np.abs(rphi).max())
    assert np.allclose(grad.cpu().numpy(), rgrad, rtol=0, atol=1e-13 * np.abs(rgrad).max())


def test_autograd_harness_on_cuda_tensors(pkg):
    """The autograd harness on CUDA tensors (device forward, device adjoint
    reusing the forward gradient) gives the host path's gradients."""
    import torch
    from fmm_autograd import fmm_potential
    x, q = uniform01(1500, 15)
    a = args(pkg, 5, 32, 1, 0)
    w = torch.tensor(np.random.default_rng(16).standard_normal(len(q)))
    xt = torch.tensor(x, device="cuda", requires_grad=True)
    qt = torch.tensor(q, device="cuda", requires_grad=True)
    phi = fmm_potential(xt, qt, pkg, a)
    (phi * w.cuda()).sum().backward()
    f = pkg.LaplaceFMM(x, q, a)
    rphi, _ = f.solve()
    dq, dx = f.adjoint(w.numpy())
    assert np.allclose(phi.detach().cpu().numpy(), rphi, rtol=0, atol=1e-12 * np.abs(rphi).max())
    assert np.allclose(qt.grad.cpu().numpy(), dq, rtol=0, atol=1e-12 * np.abs(dq).max())
    assert np.allclose(xt.grad.cpu().numpy(), dx, rtol=0, atol=1e-12 * np.abs(dx).max())
