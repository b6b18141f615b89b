"""ccsd_gpu_solve_gs_batch: independent systems of uneven size on concurrent contexts."""

import numpy as np
import pytest

from et_b200.synthetic import make_system

pytestmark = pytest.mark.gpu


def _systems(sizes):
    out = []
    for k, o in enumerate(sizes):
        s = make_system(o, 5 * o, 3 * (o + 5 * o), seed=400 + k)
        out.append(s)
    return out


@pytest.mark.parametrize("workers", [1, 3])
def test_batch_matches_single_solves(workers):
    from et_b200 import CCSD, FP64, solve_ground_states
    systems = _systems([4, 7, 5, 3, 6])
    e, it, st, ts = solve_ground_states([(s.L_mo, s.h_mo, s.eps, s.n_o, s.e_hf) for s in systems],
                                        precision=FP64, workers=workers, omega_threshold=1e-10,
                                        energy_threshold=1e-12, amplitudes=True)
    assert (st == 0).all()
    for k, s in enumerate(systems):
        with CCSD(s.n_o, s.L_mo.shape[1] - s.n_o, s.L_mo.shape[0]) as g:
            g.set_system(s.L_mo, s.h_mo, s.eps, s.e_hf)
            g.set_initial_amplitudes_guess()
            e1, it1, _, _ = g.solve_ground_state(omega_threshold=1e-10, energy_threshold=1e-12)
            assert abs(e[k] - e1) < 1e-12 and it[k] == it1
            assert np.abs(ts[k] - g.get_amplitudes()).max() < 1e-12


def test_batch_mixed_energies_and_per_system_status():
    """Mixed precision with refinement lands on the FP64 energies; a system that cannot converge
    in the iteration limit reports its own status without stopping the others."""
    from et_b200 import FP64, MIXED, solve_ground_states
    systems = _systems([8, 6, 10, 5])
    args = [(s.L_mo, s.h_mo, s.eps, s.n_o, s.e_hf) for s in systems]
    e64, _, st64, _ = solve_ground_states(args, precision=FP64, workers=4, omega_threshold=1e-9,
                                          energy_threshold=1e-11)
    em, _, stm, _ = solve_ground_states(args, precision=MIXED, workers=4, omega_threshold=1e-9,
                                        energy_threshold=1e-11, mixed_min_flops=1)
    assert (st64 == 0).all() and (stm == 0).all()
    assert np.abs(em - e64).max() < 1e-9
    e2, it2, st2, _ = solve_ground_states(args, precision=FP64, workers=2, max_iterations=3,
                                          omega_threshold=1e-12, energy_threshold=1e-14)
    assert (st2 == -5).all() and (it2 == 3).all()
