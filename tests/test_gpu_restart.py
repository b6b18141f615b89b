"""The device path against the vectors eT wrote for H2O+He/cc-pVDZ (tests/restart_ccsd_v1.0).

In eT's own MO basis: Omega(t_eT) = 0, A r = omega r, l^T A = omega l^T, A^T tbar = -eta, each to
the 1e-11 convergence of eT's run; solving from scratch on the device lands on eT's vectors.
"""

import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def et():
    from oracle import frontend as fe
    return fe.et_restart_system()


def _ctx(d, precision=0, **kw):
    from et_b200 import CCSD
    n_J, n_o = d["L_mo"].shape[0], d["n_o"]
    g = CCSD(n_o, d["h_mo"].shape[0] - n_o, n_J, precision=precision, **kw)
    g.set_system(d["L_mo"], d["h_mo"], d["eps"], d["e_hf"])
    return g


def _angle(x, y):
    c = abs(x @ y) / (np.linalg.norm(x) * np.linalg.norm(y))
    return np.sqrt(max(0.0, 1.0 - c * c))


def test_et_vectors_fp64(et):
    g = _ctx(et)
    g.set_amplitudes(et["t"])
    assert np.linalg.norm(g.construct_omega()) < 1e-10
    assert abs(g.calculate_energy() - et["e_ccsd"]) < 1e-10
    R = et["r"].T.copy()
    AR = g.jacobian_transformation(R)
    assert np.abs(AR - R * et["omega"]).max() < 1e-10
    Lv = et["l"].T.copy()
    LA = g.jacobian_transpose_transformation(Lv)
    assert np.abs(LA - Lv * et["omega"]).max() < 1e-10
    eta = g.construct_eta()
    assert np.linalg.norm(g.jacobian_transpose_transformation(et["tbar"]) + eta) < 1e-10
    g.close()


def test_et_vectors_mixed(et):
    """The same identities through the split-BF16 tensor-core GEMMs, at their accuracy."""
    from et_b200 import MIXED
    g = _ctx(et, MIXED, mixed_min_flops=1)
    g.set_amplitudes(et["t"])
    assert np.linalg.norm(g.construct_omega()) < 1e-5
    R = et["r"].T.copy()
    assert np.abs(g.jacobian_transformation(R) - R * et["omega"]).max() < 1e-5
    g.close()


def test_solve_from_mp2_reaches_et_amplitudes(et):
    g = _ctx(et)
    g.set_initial_amplitudes_guess()
    e, it, hist, rc = g.solve_ground_state(omega_threshold=1e-11, energy_threshold=1e-12)
    assert abs(e - et["e_ccsd"]) < 1e-10
    assert np.abs(g.get_amplitudes() - et["t"]).max() < 1e-9
    g.close()


def test_multipliers_reach_et_tbar(et):
    g = _ctx(et)
    g.set_amplitudes(et["t"])
    tbar, it = g.solve_multipliers(residual_threshold=1e-11)
    assert np.abs(tbar - et["tbar"]).max() < 1e-9
    g.close()


@pytest.mark.parametrize("left", [False, True])
def test_davidson_reaches_et_roots_and_vectors(et, left):
    g = _ctx(et)
    g.set_amplitudes(et["t"])
    w, X, it = g.excited_states(3, left=left, residual_threshold=1e-10, energy_threshold=1e-12, vectors=True)
    assert np.abs(w - et["omega"]).max() < 1e-10
    ref = et["l"] if left else et["r"]
    for k in range(3):
        assert _angle(X[:, k], ref[k]) < 1e-8
    g.close()


def test_restart_file_round_trip_through_device(et, tmp_path):
    """Amplitudes written by the device context in eT's layout restart another context exactly."""
    from et_b200 import restart as rs
    g = _ctx(et)
    g.set_amplitudes(et["t"])
    p = os.path.join(tmp_path, "t")
    g.save_amplitudes(p)
    v, e, n = rs.read_amplitudes(p, rs.ccsd_blocks(et["n_o"], et["L_mo"].shape[1] - et["n_o"]))
    assert np.array_equal(v, et["t"]) and abs(e - et["e_ccsd"]) < 1e-10
    h = _ctx(et)
    assert h.read_amplitudes(p) == v.size
    assert h.calculate_energy() == g.calculate_energy()
    g.close()
    h.close()
