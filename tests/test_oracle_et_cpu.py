"""The CPU restatement of eT's algorithm that the benchmark times (oracle/et_cpu.py: batched A2
ladder, OpenMP packing) equals the oracle that is pinned to eT's outputs (oracle/ccsd.py)."""

import numpy as np
import pytest

from et_b200.synthetic import make_system
from oracle import ccsd as oc
from oracle import et_cpu


@pytest.mark.parametrize("dims,batch", [((4, 16, 40), None), ((4, 16, 40), 3), ((5, 13, 37), 1),
                                        ((3, 9, 20), 4), ((1, 5, 8), 2), ((2, 1, 4), None)])
def test_batched_residual_equals_oracle(dims, batch):
    n_o, n_v, n_J = dims
    s = make_system(n_o, n_v, n_J, seed=31)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o, s.e_hf)
    et = et_cpu.ETSystem(s.L_mo, s.h_mo, s.eps, s.n_o, s.e_hf, batch=batch)
    amp = 0.05 * np.random.default_rng(2).standard_normal(ref.n_amp)
    ref.set_amplitudes(amp)
    et.set_amplitudes(amp)
    om, om_ref = et.omega(), ref.omega()
    assert np.abs(om - om_ref).max() <= 1e-13 * max(1.0, np.abs(om_ref).max())
    assert abs(et.energy() - ref.energy()) <= 1e-13
    # the literal +/- algorithm alone, against the dense ladder
    t = oc.squareup(ref.t2, ref.n_v, ref.n_o)
    a2 = et_cpu.omega_a2_batched(ref.t2, np.asfortranarray(ref.L_t1[:, n_o:, n_o:]), n_o, batch=batch)
    assert np.abs(a2 - oc.omega_ccsd_a2_dense(t, ref.L_t1, n_o)).max() <= 1e-13


def test_mp2_start_and_one_iteration_equal_oracle():
    s = make_system(4, 12, 30, seed=5)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o, s.e_hf)
    et = et_cpu.ETSystem(s.L_mo, s.h_mo, s.eps, s.n_o, s.e_hf, batch=5)
    ref.mp2_start()
    et.mp2_start()
    assert np.abs(et.get_amplitudes() - ref.get_amplitudes()).max() <= 1e-14
    for sysm in (ref, et):
        oc.solve_gs(sysm, max_iterations=2, omega_threshold=0.0, energy_threshold=-1.0)
    assert np.abs(et.get_amplitudes() - ref.get_amplitudes()).max() <= 1e-13
    assert np.abs(et.fock - ref.fock).max() <= 1e-13
