"""The CCSD residual as a torch.autograd.Function, for gradient checks of the device adjoint.

eT has no Python layer; this wrapper exists so that the adjoint behind ``ccsd_gpu_vjp`` (the
transpose Jacobian in t plus the adjoints into the Cholesky vectors and h) can be checked with
``torch.autograd.gradcheck`` against finite differences of the device residual itself:

    from et_b200.autograd import residual
    omega = residual(gpu, t, L_mo, h_mo)        # float64 tensors; gpu = et_b200.CCSD
    torch.autograd.gradcheck(lambda t, L, h: residual(gpu, t, L, h), (t, L, h))

Forward: Omega(t; L, h) at the given amplitudes and integrals (construct_omega).  Backward:
(dOmega/dt)^T b, (dOmega/dL)^T b, (dOmega/dh)^T b for the incoming cotangent b (ccsd_gpu_vjp).
Tensors travel through host memory; the arithmetic runs in libccsd_gpu.so.
"""

from __future__ import annotations

import numpy as np
import torch


class ResidualFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, gpu, eps, e_hf, t, L, h):
        tn, Ln, hn = (x.detach().cpu().double().numpy() for x in (t, L, h))
        gpu.set_system(Ln, hn, eps, e_hf)
        gpu.set_amplitudes(tn)
        om = gpu.construct_omega()
        ctx.gpu, ctx.eps, ctx.e_hf = gpu, eps, e_hf
        ctx.save_for_backward(t, L, h)
        return torch.from_numpy(om).to(t.device)

    @staticmethod
    def backward(ctx, grad):
        t, L, h = ctx.saved_tensors
        gpu = ctx.gpu
        # the context may have moved on since forward: restore the point of linearisation
        gpu.set_system(L.detach().cpu().numpy(), h.detach().cpu().numpy(), ctx.eps, ctx.e_hf)
        gpu.set_amplitudes(t.detach().cpu().numpy())
        b = grad.detach().cpu().double().numpy()
        want_L, want_h = ctx.needs_input_grad[4], ctx.needs_input_grad[5]
        out = gpu.vjp(b, want_L=want_L, want_h=want_h)
        out = list(out) if isinstance(out, tuple) else [out]
        dt = out.pop(0)
        dL = out.pop(0) if want_L else None
        dh = out.pop(0) if want_h else None

        def as_t(x, like):
            return None if x is None else torch.from_numpy(np.ascontiguousarray(x)).to(like.device)

        return None, None, None, as_t(dt, t), as_t(dL, L), as_t(dh, h)


def residual(gpu, t, L, h, eps=None, e_hf=0.0):
    """Omega(t; L, h) with gradients to t, L (J, p, q) and h through the device adjoint.

    ``eps`` (orbital energies) only enters the solvers' preconditioners, not Omega; the diagonal of
    h is used when it is not given."""
    if eps is None:
        eps = np.diag(h.detach().cpu().numpy()).copy()
    return ResidualFunction.apply(gpu, eps, e_hf, t, L, h)
