"""The device one-electron density against the oracle's and against eT's CCSD dipole moment
(tests/ccsd_dipole: H2O and He, STO-3G, Cholesky 1e-11)."""

import numpy as np
import pytest

from oracle import ccsd as oc

pytestmark = pytest.mark.gpu


def test_density_and_dipole_match_oracle_and_et():
    from et_b200 import CCSD
    from oracle import frontend as fe
    d = fe.et_dipole_system()
    n_o, n_J = d["n_o"], d["L_mo"].shape[0]
    n_v = d["h_mo"].shape[0] - n_o
    with CCSD(n_o, n_v, n_J) as g:
        g.set_system(d["L_mo"], d["h_mo"], d["eps"], d["e_hf"])
        g.set_initial_amplitudes_guess()
        e, _, _, _ = g.solve_ground_state(omega_threshold=1e-12, energy_threshold=1e-13)
        tbar, _ = g.solve_multipliers(residual_threshold=1e-12)
        D = g.one_electron_density(tbar)
        amp = g.get_amplitudes()
    ref = d["reference"]
    assert abs(e - ref["e_ccsd"]) < 1e-9
    s = oc.CCSDSystem(d["L_mo"], d["h_mo"], d["eps"], n_o, d["e_hf"])
    s.set_amplitudes(amp)
    D_ref = oc.one_electron_density(s, tbar)
    assert np.abs(D - D_ref).max() < 1e-10
    assert abs(np.trace(D) - 2 * n_o) < 1e-10
    dip = ref["dipole_debye"]
    mu_el = -np.einsum("xpq,pq->x", d["mu_mo"], D) * dip["debye_per_au"]
    # eT prints its Debye conversion factor to nine digits: ~4e-8 D of rounding at |mu| ~ 34 D
    assert np.abs(mu_el - np.array(dip["electronic"])).max() < 2e-7


def test_density_hellmann_feynman_synthetic():
    """sum V_pq D_pq is the derivative of the converged energy along h -> h + lambda V (central
    differences of full FP64 solves; the energy adds the h-dependence of the reference and of the
    singles term, which calculate_energy leaves to the caller at a Hartree-Fock reference)."""
    from et_b200 import CCSD
    from et_b200.synthetic import make_system
    n_o, n_v, n_J = 4, 12, 30
    s = make_system(n_o, n_v, n_J, seed=77)
    rng = np.random.default_rng(1)
    V = rng.standard_normal((n_o + n_v, n_o + n_v))
    V = 0.5 * (V + V.T)
    lam = 1e-4

    def solve(h):
        with CCSD(n_o, n_v, n_J) as g:
            g.set_system(s.L_mo, h, s.eps, s.e_hf)
            g.set_initial_amplitudes_guess()
            e, _, _, _ = g.solve_ground_state(omega_threshold=1e-12, energy_threshold=1e-14)
            t = g.get_amplitudes()
            return g, e, t

    with CCSD(n_o, n_v, n_J) as g:
        g.set_system(s.L_mo, s.h_mo, s.eps, s.e_hf)
        g.set_initial_amplitudes_guess()
        g.solve_ground_state(omega_threshold=1e-12, energy_threshold=1e-14)
        tbar, _ = g.solve_multipliers(residual_threshold=1e-12)
        D = g.one_electron_density(tbar)
    e_pm = []
    for sign in (1.0, -1.0):
        h = s.h_mo + sign * lam * V
        _, e, t = solve(h)
        t1 = t[: n_o * n_v].reshape(n_v, n_o, order="F")
        # h-dependence of the reference energy and of the singles term 2 sum_ai h_ia t_ai
        e += sign * lam * (2.0 * np.trace(V[:n_o, :n_o]) + 2.0 * np.sum(V[:n_o, n_o:] * t1.T))
        e_pm.append(e)
    fd = (e_pm[0] - e_pm[1]) / (2 * lam)
    assert abs(fd - np.sum(V * D)) < 1e-7 * max(1.0, abs(fd))
