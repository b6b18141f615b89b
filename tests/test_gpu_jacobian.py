"""Jacobian transformation, its transpose and the adjoint into L and h against the CPU oracle."""

import numpy as np
import pytest

from et_b200.synthetic import make_system
from oracle import ccsd as oc

pytestmark = pytest.mark.gpu


def _setup(n_o, n_v, n_J, seed=3, scale=0.05):
    from et_b200 import CCSD
    s = make_system(n_o, n_v, n_J, seed=seed)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    amp = scale * np.random.default_rng(seed + 5).standard_normal(ref.n_amp)
    ref.set_amplitudes(amp)
    gpu = CCSD(n_o, n_v, n_J)
    gpu.set_system(s.L_mo, s.h_mo, s.eps)
    gpu.set_amplitudes(amp)
    return s, ref, gpu, amp


@pytest.mark.parametrize("dims", [(2, 5, 9), (3, 8, 20), (5, 13, 30)])
def test_jacobian_matches_oracle(dims):
    s, ref, gpu, amp = _setup(*dims)
    rng = np.random.default_rng(1)
    for _ in range(2):
        c = rng.standard_normal(ref.n_amp)
        rho = gpu.jacobian_transformation(c)
        rho_ref = ref.jacobian_transformation(c)
        assert np.abs(rho - rho_ref).max() <= 1e-11 * max(1.0, np.abs(rho_ref).max())
    gpu.close()


def test_jacobian_block_of_trials():
    """n_vec trial vectors in one call equal n_vec single calls."""
    s, ref, gpu, amp = _setup(3, 9, 21)
    C = np.random.default_rng(2).standard_normal((ref.n_amp, 5))
    R = gpu.jacobian_transformation(C)
    for k in range(5):
        assert np.abs(R[:, k] - ref.jacobian_transformation(C[:, k])).max() < 1e-11 * max(1, np.abs(R).max())
    gpu.close()


def test_transpose_matches_dense_oracle():
    s, ref, gpu, amp = _setup(2, 6, 12)
    A = ref.jacobian_matrix()
    B = np.random.default_rng(3).standard_normal((ref.n_amp, 3))
    S = gpu.jacobian_transpose_transformation(B)
    assert np.abs(S - A.T @ B).max() <= 1e-11 * max(1.0, np.abs(A).max())
    gpu.close()


@pytest.mark.parametrize("dims", [(4, 12, 30), (6, 24, 60)])
def test_transpose_dot_identity(dims):
    """<b, A c> == <A^T b, c> for random b, c (size-independent property)."""
    s, ref, gpu, amp = _setup(*dims)
    rng = np.random.default_rng(4)
    b, c = rng.standard_normal(ref.n_amp), rng.standard_normal(ref.n_amp)
    lhs = b @ gpu.jacobian_transformation(c)
    rhs = gpu.jacobian_transpose_transformation(b) @ c
    assert abs(lhs - rhs) <= 1e-11 * max(1.0, abs(lhs))
    gpu.close()


def _omega_complex(L, h, amp, n_o):
    n_v = h.shape[0] - n_o
    n_t1 = n_o * n_v
    t1 = amp[:n_t1].reshape(n_v, n_o, order="F")
    L_t1 = oc.construct_t1_cholesky(L, t1, n_o)
    F = oc.construct_fock(h, L_t1, t1, n_o)
    return oc.omega_ccsd(t1, amp[n_t1:], L, L_t1, F, n_o)


def test_adjoint_into_cholesky_vectors_and_h():
    """<dL, dL_dir> + <dh, dh_dir> == b^T (dOmega/d(L,h))(dir) by complex-step differentiation."""
    s, ref, gpu, amp = _setup(3, 7, 15)
    rng = np.random.default_rng(6)
    b = rng.standard_normal(ref.n_amp)
    dt, dL, dh = gpu.vjp(b, want_L=True, want_h=True)
    # amplitude part: D (dOmega/dt)^T b is the transpose transformation
    sig = gpu.jacobian_transpose_transformation(b)
    assert np.abs(dt * ref.diag_scaling() - sig).max() < 1e-11 * max(1.0, np.abs(sig).max())
    dLdir = rng.standard_normal(s.L_mo.shape)
    dhdir = rng.standard_normal(s.h_mo.shape)
    hstep = 1e-30
    om_L = _omega_complex(s.L_mo + 1j * hstep * dLdir, s.h_mo.astype(complex), amp, s.n_o)
    om_h = _omega_complex(s.L_mo.astype(complex), s.h_mo + 1j * hstep * dhdir, amp, s.n_o)
    ref_L = b @ (np.imag(om_L) / hstep)
    ref_h = b @ (np.imag(om_h) / hstep)
    assert abs(np.sum(dL * dLdir) - ref_L) <= 1e-10 * max(1.0, abs(ref_L))
    assert abs(np.sum(dh * dhdir) - ref_h) <= 1e-10 * max(1.0, abs(ref_h))
    gpu.close()


def test_excitation_energies_match_et(h2o_he):
    """Davidson on the CPU using the GPU Jacobian reproduces eT's EOM-CCSD roots (H2O+He)."""
    from et_b200 import CCSD
    from oracle import frontend as fe
    d = h2o_he
    n_J, n_o = d["L_mo"].shape[0], d["n_o"]
    gpu = CCSD(n_o, d["h_mo"].shape[0] - n_o, n_J)
    gpu.set_system(d["L_mo"], d["h_mo"], d["eps"], d["e_hf"])
    gpu.set_initial_amplitudes_guess()
    gpu.solve_ground_state(omega_threshold=1e-11, energy_threshold=1e-12)

    class GpuA:
        def __init__(self):
            s = oc.CCSDSystem(d["L_mo"], d["h_mo"], d["eps"], n_o, d["e_hf"])
            self.n_amp, self._eps = s.n_amp, s.orbital_differences()

        def orbital_differences(self):
            return self._eps

        def jacobian_transformation(self, c):
            return gpu.jacobian_transformation(c)

    w, _, _ = oc.davidson_right(GpuA(), 2, threshold=1e-9)
    ref = fe.golden_values()["ccsd_right_es_energies"]["excitation_energies"]
    assert np.allclose(w, ref, atol=1e-10)
    gpu.close()


@pytest.mark.parametrize("left", [False, True])
def test_device_davidson_matches_et(h2o_he, left):
    """eigen_davidson_solver on the device (right and left) reproduces eT's EOM-CCSD roots."""
    from et_b200 import CCSD
    from oracle import frontend as fe
    d = h2o_he
    n_J, n_o = d["L_mo"].shape[0], d["n_o"]
    gpu = CCSD(n_o, d["h_mo"].shape[0] - n_o, n_J)
    gpu.set_system(d["L_mo"], d["h_mo"], d["eps"], d["e_hf"])
    gpu.set_initial_amplitudes_guess()
    gpu.solve_ground_state(omega_threshold=1e-11, energy_threshold=1e-12)
    w, X, it = gpu.excited_states(2, left=left, residual_threshold=1e-9, energy_threshold=1e-11, vectors=True)
    name = "ccsd_left_es_energies" if left else "ccsd_right_es_energies"
    ref = fe.golden_values()[name]["excitation_energies"]
    assert np.allclose(w, ref, atol=1e-10), (w, ref)
    # eigenvector property checked through the transformation itself
    AX = gpu.jacobian_transpose_transformation(X) if left else gpu.jacobian_transformation(X)
    assert np.abs(AX - X * w).max() < 1e-8
    gpu.close()


def test_device_davidson_block_matches_oracle():
    """A block of trial vectors transformed per call (block=3) on a synthetic system."""
    s, ref, gpu, amp = _setup(4, 12, 30, scale=0.0)
    ref.mp2_start()
    gpu.set_initial_amplitudes_guess()
    w_ref, _, _ = oc.davidson_right(ref, 3, threshold=1e-9)
    w, _, _ = gpu.excited_states(3, block=3, residual_threshold=1e-9, energy_threshold=1e-11)
    assert np.allclose(np.sort(w), np.sort(w_ref), atol=1e-9)
    gpu.close()


def test_eta_matches_oracle():
    s, ref, gpu, amp = _setup(3, 8, 20)
    eta = gpu.construct_eta()
    eta_ref = oc.construct_eta(ref.fock, ref.L_t1, ref.n_o)
    assert np.abs(eta - eta_ref).max() < 1e-12 * max(1.0, np.abs(eta_ref).max())
    gpu.close()


def test_multipliers_match_dense_oracle_solve():
    """Lambda equations A^T tbar = -eta at the ground-state solution vs a dense oracle solve."""
    from et_b200 import CCSD
    n_o, n_v, n_J = 3, 8, 20
    s = make_system(n_o, n_v, n_J, seed=17)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    ref.mp2_start()
    oc.solve_gs(ref, omega_threshold=1e-11, energy_threshold=1e-13)
    gpu = CCSD(n_o, n_v, n_J)
    gpu.set_system(s.L_mo, s.h_mo, s.eps)
    gpu.set_amplitudes(ref.get_amplitudes())
    tbar, it = gpu.solve_multipliers(residual_threshold=1e-10)
    A = ref.jacobian_matrix()
    eta = oc.construct_eta(ref.fock, ref.L_t1, ref.n_o)
    tbar_ref = np.linalg.solve(A.T, -eta)
    assert np.abs(tbar - tbar_ref).max() < 1e-8 * max(1.0, np.abs(tbar_ref).max())
    gpu.close()


def test_multipliers_residual_h2o_he(h2o_he):
    from et_b200 import CCSD
    d = h2o_he
    n_J, n_o = d["L_mo"].shape[0], d["n_o"]
    gpu = CCSD(n_o, d["h_mo"].shape[0] - n_o, n_J)
    gpu.set_system(d["L_mo"], d["h_mo"], d["eps"], d["e_hf"])
    gpu.set_initial_amplitudes_guess()
    gpu.solve_ground_state(omega_threshold=1e-10, energy_threshold=1e-12)
    tbar, it = gpu.solve_multipliers(residual_threshold=1e-9)
    r = gpu.jacobian_transpose_transformation(tbar) + gpu.construct_eta()
    assert np.linalg.norm(r) < 1e-8
    gpu.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_prepared_transformations_equal_fresh_ones(precision):
    """ccsd_gpu_prepare_jacobian records the residual once; the transformations that follow reuse
    it and must give exactly what a fresh recording gives.  New amplitudes drop the preparation."""
    from et_b200 import CCSD
    n_o, n_v, n_J = 4, 16, 40
    s = make_system(n_o, n_v, n_J, seed=17)
    rng = np.random.default_rng(8)
    with CCSD(n_o, n_v, n_J, precision=precision, mixed_min_flops=1) as g:
        g.set_system(s.L_mo, s.h_mo, s.eps)
        amp = 0.05 * rng.standard_normal(g.n_amp)
        g.set_amplitudes(amp)
        C = rng.standard_normal((g.n_amp, 3))
        fresh = (g.jacobian_transformation(C), g.jacobian_transpose_transformation(C))
        fresh1 = g.jacobian_transformation(C[:, 1])      # one vector: other GEMM shapes than the block
        g.prepare_for_jacobian(0)
        for _ in range(2):
            prepared = (g.jacobian_transformation(C), g.jacobian_transpose_transformation(C))
            for a, b in zip(fresh, prepared):
                assert np.array_equal(a, b)
        assert np.array_equal(g.jacobian_transformation(C[:, 1]), fresh1)
        g.set_amplitudes(2.0 * amp)
        ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
        ref.set_amplitudes(2.0 * amp)
        rho, rho_ref = g.jacobian_transformation(C[:, 0]), ref.jacobian_transformation(C[:, 0])
        tol = 1e-11 if precision == 0 else 1e-4
        assert np.linalg.norm(rho - rho_ref) <= tol * np.linalg.norm(rho_ref)
        g.prepare_for_jacobian(1)
        g.prepare_for_jacobian(-1)
