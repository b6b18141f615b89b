"""Oracle pinned to the vectors eT wrote (tests/restart_ccsd_v1.0), and the restart-file I/O.

eT converged t, tbar and the EOM vectors to 1e-11 with a 1e-12 Cholesky threshold; in eT's own
MO basis the restated residual, Jacobian, transpose and eta must annihilate them to that level.
"""

import os

import numpy as np
import pytest

from et_b200 import restart as rs
from oracle import ccsd as oc


@pytest.fixture(scope="module")
def et_restart():
    from oracle import frontend as fe
    d = fe.et_restart_system()
    s = oc.CCSDSystem(d["L_mo"], d["h_mo"], d["eps"], d["n_o"], d["e_hf"])
    s.set_amplitudes(d["t"])
    return d, s


def test_ao_conventions_match_et(et_restart):
    """eT's MO coefficients are orthonormal in this AO basis (same order, normalisation and phases)."""
    d, _ = et_restart
    C, S = d["C"], d["S"]
    assert np.abs(C.T @ S @ C - np.eye(C.shape[1])).max() < 1e-13


def test_fock_reproduces_et_orbital_energies(et_restart):
    d, s = et_restart
    z = oc.CCSDSystem(d["L_mo"], d["h_mo"], d["eps"], d["n_o"], d["e_hf"])
    F = z.fock
    assert np.abs(np.diag(F) - d["eps"]).max() < 1e-10
    assert np.abs(F - np.diag(np.diag(F))).max() < 1e-10


def test_et_amplitudes_solve_the_restated_equations(et_restart):
    d, s = et_restart
    assert np.linalg.norm(s.omega()) < 1e-10
    assert abs(s.energy() - d["e_ccsd"]) < 1e-10


def test_et_right_vectors_are_eigenvectors(et_restart):
    d, s = et_restart
    for r, w in zip(d["r"], d["omega"]):
        assert np.linalg.norm(s.jacobian_transformation(r) - w * r) < 1e-10


def test_et_left_vectors_and_multipliers_by_projection(et_restart):
    """l^T A = omega l^T and A^T tbar = -eta, tested on random directions x through A x."""
    d, s = et_restart
    eta = oc.construct_eta(s.fock, s.L_t1, s.n_o)
    rng = np.random.default_rng(11)
    for _ in range(3):
        x = rng.standard_normal(s.n_amp)
        Ax = s.jacobian_transformation(x)
        assert abs(d["tbar"] @ Ax + eta @ x) < 1e-9
        for l, w in zip(d["l"], d["omega"]):
            assert abs(l @ Ax - w * (l @ x)) < 1e-9
    # the stored pairs are biorthonormal
    assert np.abs(d["l"] @ d["r"].T - np.eye(3)).max() < 1e-10


def test_restart_round_trip(tmp_path, et_restart):
    d, s = et_restart
    blocks = rs.ccsd_blocks(s.n_o, s.n_v)
    p = os.path.join(tmp_path, "t")
    rs.save_amplitudes(p, d["t"], blocks, energy=d["e_ccsd"])
    assert os.path.getsize(p) == 8 + 8 * len(blocks) + 8 * sum(blocks)
    v, e, n = rs.read_amplitudes(p, blocks)
    assert np.array_equal(v, d["t"]) and e == d["e_ccsd"] and n == sum(blocks)


def test_restart_singles_only_and_wrong_size(tmp_path):
    blocks = rs.ccsd_blocks(2, 3)
    p = os.path.join(tmp_path, "t")
    rs.save_amplitudes(p, np.arange(6.0), [6], energy=-1.5)          # CCS singles only
    v, e, n = rs.read_amplitudes(p, blocks)
    assert n == 6 and e == -1.5 and np.array_equal(v[:6], np.arange(6.0)) and not v[6:].any()
    rs.save_amplitudes(p, np.arange(7.0), [7])
    with pytest.raises(rs.RestartFileError):
        rs.read_amplitudes(p, blocks)


def test_legacy_directory_conversion(tmp_path):
    """An eT 1.0 directory (record files) converts to the current layout."""
    n_o, n_v = 2, 3
    n1, n2 = 6, 21
    old, new = os.path.join(tmp_path, "old"), os.path.join(tmp_path, "new")
    os.makedirs(old)
    rng = np.random.default_rng(0)
    t = rng.standard_normal(n1 + n2)
    r = rng.standard_normal(n1 + n2)
    i8 = lambda x: np.array([x], dtype="<i8").tobytes()
    rs.write_records(os.path.join(old, "cc_restart_file"), [i8(n_o), i8(n_v), i8(n1 + n2), i8(n1 + n2)])
    rs.write_records(os.path.join(old, "t"), [t[:n1].tobytes(), t[n1:].tobytes()])
    rs.write_records(os.path.join(old, "r_001"), [r.tobytes()])
    rs.write_records(os.path.join(old, "excitation_energies"), [i8(1), np.array([0.25]).tobytes()])
    written = rs.convert_legacy_directory(old, new)
    assert sorted(written) == ["r_001", "t"]
    v, e, _ = rs.read_amplitudes(os.path.join(new, "t"), [n1, n2])
    assert np.array_equal(v, t) and e == 0.0
    v, e, _ = rs.read_amplitudes(os.path.join(new, "r_001"), [n1, n2])
    assert np.array_equal(v, r) and e == 0.25
    with open(os.path.join(old, "bad"), "wb") as f:
        f.write((16).to_bytes(4, "little") + bytes(16) + (8).to_bytes(4, "little"))
    with pytest.raises(rs.RestartFileError):
        rs.read_records(os.path.join(old, "bad"))
