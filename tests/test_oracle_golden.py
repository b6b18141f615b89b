"""The CPU oracle against eT's own committed regression outputs (no GPU)."""

import numpy as np
import pytest

from oracle import ccsd as oc
from oracle import frontend as fe


def _system(d):
    return oc.CCSDSystem(d["L_mo"], d["h_mo"], d["eps"], d["n_o"], d["e_hf"])


def test_hf_and_cholesky_match_et(h2o_he):
    ref = fe.golden_values()["ccsd_gs_energy"]
    assert abs(h2o_he["e_hf"] - ref["e_hf"]) < 1e-9
    assert h2o_he["L_mo"].shape[0] == ref["n_cholesky"]
    # the T1 Fock matrix at t1 = 0 is the canonical (diagonal) HF Fock matrix
    s = _system(h2o_he)
    assert np.abs(s.fock - np.diag(h2o_he["eps"])).max() < 1e-9


def test_ccsd_iteration_history_matches_et(h2o_he):
    """Every (E, |Omega|) pair of eT's DIIS/quasi-Newton run (tests/ccsd_gs_energy)."""
    ref = fe.golden_values()["ccsd_gs_energy"]
    s = _system(h2o_he)
    s.mp2_start()
    hist = []
    e, it, conv = oc.solve_gs(s, history=hist)
    assert conv and it == len(ref["gs_history"])
    for (E, n), (E_ref, n_ref) in zip(hist, ref["gs_history"]):
        assert abs(E - E_ref) < 2e-12
        ulp = 10.0 ** (np.floor(np.log10(n_ref)) - 3)     # eT prints |Omega| as 0.dddd E+xx
        assert abs(n - n_ref) <= 0.51 * ulp
    assert abs(e - ref["e_ccsd"]) < 1e-10


def test_water_ccsd_matches_et():
    ref = fe.golden_values()["ccsd_lr_polarizability"]
    d = fe.et_test_system("ccsd_lr_polarizability")
    assert d["L_mo"].shape[0] == ref["n_cholesky"]
    assert abs(d["e_hf"] - ref["e_hf"]) < 1e-9
    s = _system(d)
    s.mp2_start()
    e, it, conv = oc.solve_gs(s)
    assert conv and abs(e - ref["e_ccsd"]) < 1e-10


@pytest.mark.slow
def test_excitation_energies_match_et(h2o_he):
    """Right Jacobian A = (dOmega/dt) D pinned by eT's EOM-CCSD roots (left == right)."""
    vals = fe.golden_values()
    s = _system(h2o_he)
    s.mp2_start()
    oc.solve_gs(s)
    w, X, _ = oc.davidson_right(s, 2, threshold=1e-10)
    for ref_name in ("ccsd_right_es_energies", "ccsd_left_es_energies"):
        ref = vals[ref_name]["excitation_energies"]
        assert np.allclose(w, ref, atol=2e-12)


def test_ladder_pm_algorithm_equals_dense():
    """eT's +/- A2 algorithm and its dense restatement agree."""
    from et_b200.synthetic import make_system
    sy = make_system(3, 6, 15, seed=3)
    s = oc.CCSDSystem(sy.L_mo, sy.h_mo, sy.eps, sy.n_o)
    amp = 0.05 * np.random.default_rng(0).standard_normal(s.n_amp)
    s.set_amplitudes(amp)
    assert np.abs(s.omega() - s.omega(ladder="pm")).max() < 1e-14


def test_packing_roundtrip():
    n_v, n_o = 5, 3
    x = np.random.default_rng(1).standard_normal(oc.n_t2(n_o, n_v))
    full = oc.squareup(x, n_v, n_o)
    assert np.allclose(full, np.einsum("aibj->bjai", full))
    assert np.array_equal(oc.packin(full, n_v, n_o), x)
