"""torch.autograd.Function over the C ABI (test harness only).

forward:  phi = FMM(x, q) (potential at the bodies, input order)
backward: for an upstream weight w = dL/dphi, the library's adjoint gives
          dL/dq and dL/dx.

CPU tensors go through the host-buffer calls (rtfmm_b200_solve,
rtfmm_b200_adjoint).  CUDA tensors stay on the device: the tree is built from
a host copy of the positions, then the charges, the potential, the weights
and both gradients move through rtfmm_b200_forward_device and
rtfmm_b200_adjoint_device, which reuses the forward pass's gradient.
"""
import numpy as np
import torch


class FMMPotential(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, q, pkg, args):
        xn = x.detach().cpu().numpy().astype(np.float64)
        if x.is_cuda:
            qd = q.detach().to(torch.float64).contiguous()
            f = pkg.LaplaceFMM(xn, qd.cpu().numpy(), args)
            f.setup()
            f.upload()
            phi = torch.empty(len(qd), dtype=torch.float64, device=x.device)
            f.forward_device(qd.data_ptr(), phi.data_ptr(), 0)
            ctx.fmm = f
            ctx.dtype = x.dtype
            return phi.to(x.dtype)
        qn = q.detach().cpu().numpy().astype(np.float64)
        f = pkg.LaplaceFMM(xn, qn, args)
        phi, _ = f.solve()
        ctx.fmm = f
        ctx.dtype = x.dtype
        return torch.from_numpy(phi).to(x.device)

    @staticmethod
    def backward(ctx, grad_phi):
        dev = grad_phi.device
        if grad_phi.is_cuda:
            w = grad_phi.detach().to(torch.float64).contiguous()
            dq = torch.empty_like(w)
            dx = torch.empty((len(w), 3), dtype=torch.float64, device=dev)
            ctx.fmm.adjoint_device(w.data_ptr(), dq.data_ptr(), dx.data_ptr())
            ctx.fmm.close()
            return dx.to(ctx.dtype), dq.to(ctx.dtype), None, None
        w = grad_phi.detach().cpu().numpy().astype(np.float64)
        dq, dx = ctx.fmm.adjoint(w)
        ctx.fmm.close()
        return (torch.from_numpy(dx).to(dev, ctx.dtype), torch.from_numpy(dq).to(dev, ctx.dtype), None, None)


def fmm_potential(x, q, pkg, args):
    return FMMPotential.apply(x, q, pkg, args)
