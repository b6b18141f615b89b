"""The oracle's unrelaxed CCSD one-electron density against eT's ground-state dipole moment
(tests/ccsd_dipole: H2O and He, STO-3G, Cholesky 1e-11, converged to 1e-11).

The density is d(E + tbar^T Omega)/dh at the converged amplitudes and multipliers; contracted with
the dipole integrals it gives the electronic dipole moment eT prints."""

import numpy as np
import pytest

from oracle import ccsd as oc


@pytest.fixture(scope="module")
def dipole_case():
    from oracle import frontend as fe
    d = fe.et_dipole_system()
    s = oc.CCSDSystem(d["L_mo"], d["h_mo"], d["eps"], d["n_o"], d["e_hf"])
    s.mp2_start()
    oc.solve_gs(s, omega_threshold=1e-12, energy_threshold=1e-13)
    A = s.jacobian_matrix()
    eta = oc.construct_eta(s.fock, s.L_t1, s.n_o)
    tbar = np.linalg.solve(A.T, -eta)
    return d, s, tbar


def test_reference_and_ccsd_energies_match_et(dipole_case):
    d, s, _ = dipole_case
    ref = d["reference"]
    assert abs(d["e_hf"] - ref["e_hf"]) < 1e-9
    assert abs(s.energy() - ref["e_ccsd"]) < 1e-9


def test_nuclear_dipole_matches_et(dipole_case):
    d, _, _ = dipole_case
    dip = d["reference"]["dipole_debye"]
    # eT prints its Debye conversion factor to nine digits: ~4e-8 D of rounding at |mu| ~ 34 D
    assert np.abs(d["nuclear_dipole"] * dip["debye_per_au"] - np.array(dip["nuclear"])).max() < 1e-7


def test_ccsd_electronic_dipole_matches_et(dipole_case):
    d, s, tbar = dipole_case
    D = oc.one_electron_density(s, tbar)
    mu_el = -np.einsum("xpq,pq->x", d["mu_mo"], D)
    dip = d["reference"]["dipole_debye"]
    assert np.abs(mu_el * dip["debye_per_au"] - np.array(dip["electronic"])).max() < 2e-7
    # trace of the density = number of electrons
    assert abs(np.trace(D) - 2 * s.n_o) < 1e-10
