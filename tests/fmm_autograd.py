"""torch.autograd.Function over the C ABI (test harness only).

forward:  phi = FMM(x, q) (potential at the bodies, input order)
backward: for an upstream weight w = dL/dphi, the library's adjoint gives
          dL/dq and dL/dx (rtfmm_b200_adjoint).
"""
import numpy as np
import torch


class FMMPotential(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, q, pkg, args):
        xn = x.detach().cpu().numpy().astype(np.float64)
        qn = q.detach().cpu().numpy().astype(np.float64)
        f = pkg.LaplaceFMM(xn, qn, args)
        phi, _ = f.solve()
        ctx.fmm = f
        ctx.dtype = x.dtype
        return torch.from_numpy(phi).to(x.device)

    @staticmethod
    def backward(ctx, grad_phi):
        w = grad_phi.detach().cpu().numpy().astype(np.float64)
        dq, dx = ctx.fmm.adjoint(w)
        ctx.fmm.close()
        dev = grad_phi.device
        return (torch.from_numpy(dx).to(dev, ctx.dtype), torch.from_numpy(dq).to(dev, ctx.dtype), None, None)


def fmm_potential(x, q, pkg, args):
    return FMMPotential.apply(x, q, pkg, args)
