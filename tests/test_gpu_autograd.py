"""The device adjoint behind torch.autograd: gradcheck of Omega(t; L, h) against central finite
differences of the device residual, and backward() against the oracle's dense Jacobian."""

import numpy as np
import pytest
import torch

from et_b200.synthetic import make_system
from oracle import ccsd as oc

pytestmark = pytest.mark.gpu


def _inputs(n_o, n_v, n_J, seed=11, scale=0.05):
    from et_b200 import CCSD
    s = make_system(n_o, n_v, n_J, seed=seed)
    gpu = CCSD(n_o, n_v, n_J)
    amp = scale * np.random.default_rng(seed + 1).standard_normal(gpu.n_amp)
    t = torch.tensor(amp, dtype=torch.float64, requires_grad=True)
    L = torch.tensor(s.L_mo, dtype=torch.float64, requires_grad=True)
    h = torch.tensor(s.h_mo, dtype=torch.float64, requires_grad=True)
    return s, gpu, t, L, h


def test_gradcheck_amplitudes_cholesky_vectors_and_h():
    from et_b200.autograd import residual
    s, gpu, t, L, h = _inputs(2, 4, 6)
    eps = s.eps
    assert torch.autograd.gradcheck(lambda t, L, h: residual(gpu, t, L, h, eps=eps), (t, L, h),
                                    eps=1e-6, atol=1e-7, rtol=1e-5)
    gpu.close()


def test_gradcheck_fast_mode_larger():
    """Random-projection gradcheck (one directional derivative per input) at a size where the full
    numerical Jacobian would be slow."""
    from et_b200.autograd import residual
    s, gpu, t, L, h = _inputs(4, 12, 30)
    eps = s.eps
    assert torch.autograd.gradcheck(lambda t, L, h: residual(gpu, t, L, h, eps=eps), (t, L, h),
                                    eps=1e-6, atol=1e-7, rtol=1e-5, fast_mode=True)
    gpu.close()


def test_backward_in_t_is_transpose_of_oracle_jacobian():
    from et_b200.autograd import residual
    s, gpu, t, L, h = _inputs(3, 6, 12)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    ref.set_amplitudes(t.detach().numpy())
    # the oracle's Jacobian carries the doubles-diagonal scaling D: dOmega/dt = A D^-1
    dOmega_dt = ref.jacobian_matrix() / ref.diag_scaling()[None, :]
    b = torch.tensor(np.random.default_rng(2).standard_normal(gpu.n_amp))
    om = residual(gpu, t, L.detach(), h.detach(), eps=s.eps)
    (g,) = torch.autograd.grad(om, t, b)
    want = dOmega_dt.T @ b.numpy()
    assert np.abs(g.numpy() - want).max() <= 1e-11 * max(1.0, np.abs(want).max())
    # forward equals the oracle's residual at the same point
    assert np.abs(om.detach().numpy() - ref.omega()).max() <= 1e-12 * max(1.0, np.abs(ref.omega()).max())
    gpu.close()
