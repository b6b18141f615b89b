"""Host logic of et_b200.autograd without a GPU: the autograd.Function's argument routing, the
restore-before-backward step and the returned gradient slots, driven by an oracle-backed stand-in
for the device context (amplitude gradients only)."""

import numpy as np
import torch

from et_b200.synthetic import make_system
from oracle import ccsd as oc


class OracleContext:
    """The four calls the autograd wrapper makes, answered by the CPU oracle."""

    def __init__(self, n_o, n_v):
        self.n_o, self.n_v = n_o, n_v
        self.sys = None
        self.calls = []

    def set_system(self, L, h, eps, e_hf=0.0):
        self.calls.append("set_system")
        self.sys = oc.CCSDSystem(np.array(L), np.array(h), np.array(eps), self.n_o, e_hf)
        self.n_amp = self.sys.n_amp

    def set_amplitudes(self, t):
        self.calls.append("set_amplitudes")
        self.sys.set_amplitudes(np.array(t))

    def construct_omega(self):
        return self.sys.omega()

    def vjp(self, b, *, want_L=False, want_h=False):
        assert not want_L and not want_h
        self.calls.append("vjp")
        dOmega_dt = self.sys.jacobian_matrix() / self.sys.diag_scaling()[None, :]
        return dOmega_dt.T @ b


def test_gradcheck_through_oracle_context():
    from et_b200.autograd import residual
    s = make_system(2, 3, 5, seed=4)
    ctx = OracleContext(2, 3)
    ctx.set_system(s.L_mo, s.h_mo, s.eps)
    t = torch.tensor(0.05 * np.random.default_rng(1).standard_normal(ctx.n_amp), requires_grad=True)
    L = torch.tensor(s.L_mo)
    h = torch.tensor(s.h_mo)
    assert torch.autograd.gradcheck(lambda t: residual(ctx, t, L, h, eps=s.eps), (t,), eps=1e-6, atol=1e-8)


def test_backward_restores_the_point_of_linearisation():
    """A forward at another point between forward and backward must not change the gradient."""
    from et_b200.autograd import residual
    s = make_system(2, 3, 5, seed=6)
    ctx = OracleContext(2, 3)
    ctx.set_system(s.L_mo, s.h_mo, s.eps)
    rng = np.random.default_rng(3)
    t = torch.tensor(0.05 * rng.standard_normal(ctx.n_amp), requires_grad=True)
    L, h = torch.tensor(s.L_mo), torch.tensor(s.h_mo)
    om = residual(ctx, t, L, h, eps=s.eps)
    b = torch.tensor(rng.standard_normal(ctx.n_amp))
    residual(ctx, torch.zeros_like(t), L, h, eps=s.eps)  # moves the context elsewhere
    (g,) = torch.autograd.grad(om, t, b)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, 2)
    ref.set_amplitudes(t.detach().numpy())
    want = (ref.jacobian_matrix() / ref.diag_scaling()[None, :]).T @ b.numpy()
    assert np.abs(g.numpy() - want).max() < 1e-11 * max(1.0, np.abs(want).max())
    assert ctx.calls[-3:] == ["set_system", "set_amplitudes", "vjp"]
