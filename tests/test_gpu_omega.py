"""CUDA path (through the C ABI) against the CPU oracle: T1 Fock, energy, Omega, MP2 guess, solver."""

import numpy as np
import pytest

from et_b200.synthetic import make_system
from oracle import ccsd as oc
from oracle import frontend as fe

pytestmark = pytest.mark.gpu


def _pair(n_o, n_v, n_J, seed=7, amp_scale=0.05, **kw):
    from et_b200 import CCSD
    s = make_system(n_o, n_v, n_J, seed=seed)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o, s.e_hf)
    gpu = CCSD(n_o, n_v, n_J, **kw)
    gpu.set_system(s.L_mo, s.h_mo, s.eps, s.e_hf)
    rng = np.random.default_rng(seed + 1)
    amp = amp_scale * rng.standard_normal(ref.n_amp)
    ref.set_amplitudes(amp)
    gpu.set_amplitudes(amp)
    return ref, gpu, amp


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("dims", [(3, 8, 20), (5, 13, 37), (8, 40, 100)])
def test_fock_energy_omega_fp64(dims):
    ref, gpu, _ = _pair(*dims)
    assert _rel(gpu.get_fock(), ref.fock) < 1e-13
    assert abs(gpu.calculate_energy() - ref.energy()) < 1e-12 * max(1.0, abs(ref.energy()))
    om = gpu.construct_omega()
    assert _rel(om, ref.omega()) < 1e-12
    gpu.close()


@pytest.mark.parametrize("batch", [1, 2, 3, 7])
def test_forced_ladder_batching(batch):
    """Analogue of eT's ENABLE_FORCED_BATCHING: any a-batch length gives the same Omega."""
    ref, gpu, amp = _pair(4, 11, 30, ladder_batch=batch)
    assert _rel(gpu.construct_omega(), ref.omega()) < 1e-12
    gpu.close()


def test_mp2_guess_matches_oracle():
    from et_b200 import CCSD
    s = make_system(4, 12, 30, seed=11)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    ref.mp2_start()
    gpu = CCSD(4, 12, 30)
    gpu.set_system(s.L_mo, s.h_mo, s.eps)
    gpu.set_initial_amplitudes_guess()
    assert _rel(gpu.get_amplitudes(), ref.get_amplitudes()) < 1e-13
    gpu.close()


def test_ground_state_history_matches_et(h2o_he):
    """Device-resident QN + DIIS reproduces eT's tests/ccsd_gs_energy run iteration by iteration."""
    from et_b200 import CCSD
    golden = fe.golden_values()["ccsd_gs_energy"]
    d = h2o_he
    n_J = d["L_mo"].shape[0]
    n_o = d["n_o"]
    n_v = d["h_mo"].shape[0] - n_o
    gpu = CCSD(n_o, n_v, n_J)
    gpu.set_system(d["L_mo"], d["h_mo"], d["eps"], d["e_hf"])
    gpu.set_initial_amplitudes_guess()
    e, it, hist, rc = gpu.solve_ground_state(omega_threshold=1e-10, energy_threshold=1e-10)
    assert rc == 0 and it == len(golden["gs_history"])
    for (E, n), (E_ref, n_ref) in zip(hist, golden["gs_history"]):
        assert abs(E - E_ref) < 1e-11
        ulp = 10.0 ** (np.floor(np.log10(n_ref)) - 3)
        assert abs(n - n_ref) <= 0.51 * ulp
    assert abs(e - golden["e_ccsd"]) < 1e-10
    gpu.close()


def test_water_fp64_drop_in():
    """The plain-FP64 drop-in workload: H2O/cc-pVDZ, Cholesky 1e-8, residual 1e-8, vs the oracle."""
    from et_b200 import CCSD
    d = fe.water_system()
    ref = oc.CCSDSystem(d["L_mo"], d["h_mo"], d["eps"], d["n_o"], d["e_hf"])
    ref.mp2_start()
    e_ref, _, _ = oc.solve_gs(ref, omega_threshold=1e-8, energy_threshold=1e-10)
    n_J, n_o = d["L_mo"].shape[0], d["n_o"]
    gpu = CCSD(n_o, d["h_mo"].shape[0] - n_o, n_J)
    gpu.set_system(d["L_mo"], d["h_mo"], d["eps"], d["e_hf"])
    gpu.set_initial_amplitudes_guess()
    e, it, hist, rc = gpu.solve_ground_state(omega_threshold=1e-8, energy_threshold=1e-10)
    assert rc == 0 and abs(e - e_ref) < 1e-10
    gpu.close()


def test_omega_residual_vanishes_at_solution(h2o_he):
    """Size-independent property: |Omega(t*)| is at the convergence threshold after the solve."""
    from et_b200 import CCSD
    d = h2o_he
    n_J, n_o = d["L_mo"].shape[0], d["n_o"]
    gpu = CCSD(n_o, d["h_mo"].shape[0] - n_o, n_J)
    gpu.set_system(d["L_mo"], d["h_mo"], d["eps"], d["e_hf"])
    gpu.set_initial_amplitudes_guess()
    gpu.solve_ground_state(omega_threshold=1e-9, energy_threshold=1e-10)
    assert np.linalg.norm(gpu.construct_omega()) < 1e-9
    gpu.close()


def test_errors_are_status_codes():
    from et_b200 import CCSD, CCSDGPUError
    gpu = CCSD(2, 3, 4)
    with pytest.raises(CCSDGPUError) as ei:
        gpu.construct_omega()            # nothing set yet
    assert ei.value.code == -4
    with pytest.raises(ValueError):
        gpu.set_amplitudes(np.zeros(3))
    gpu.close()


@pytest.mark.parametrize("dims", [(1, 1, 2), (1, 4, 5), (4, 1, 6), (2, 3, 1), (1, 70, 40), (9, 2, 30)])
def test_extreme_shapes_fp64_and_mixed(dims):
    """Edge shapes: a single occupied or virtual orbital, a single Cholesky vector, and shapes whose
    padding to the tensor-core tiles dominates (mixed with every GEMM forced onto the tensor cores)."""
    from et_b200 import CCSD, MIXED
    n_o, n_v, n_J = dims
    s = make_system(n_o, n_v, n_J, seed=5)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    ref.set_amplitudes(0.05 * np.random.default_rng(1).standard_normal(ref.n_amp))
    om_ref = ref.omega()
    scale = max(1.0, np.abs(om_ref).max())
    for prec, tol in ((0, 1e-12), (MIXED, 1e-4)):
        with CCSD(n_o, n_v, n_J, precision=prec, mixed_min_flops=1) as gpu:
            gpu.set_system(s.L_mo, s.h_mo, s.eps)
            gpu.set_amplitudes(ref.get_amplitudes())
            assert abs(gpu.calculate_energy() - ref.energy()) <= tol * max(1.0, abs(ref.energy()))
            assert np.abs(gpu.construct_omega() - om_ref).max() <= tol * scale
            c = np.random.default_rng(2).standard_normal(ref.n_amp)
            rho_ref = ref.jacobian_transformation(c)
            assert np.abs(gpu.jacobian_transformation(c) - rho_ref).max() <= tol * max(1.0, np.abs(rho_ref).max())
