"""Per-term device timing log under eT's timing labels (ccsd_gpu_set_term_timing)."""

import pytest

from et_b200.synthetic import make_system

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_term_log_records_the_residual_and_transformation_terms(precision):
    from et_b200 import CCSD
    n_o, n_v, n_J = 4, 24, 60
    s = make_system(n_o, n_v, n_J, seed=3)
    with CCSD(n_o, n_v, n_J, precision=precision, mixed_min_flops=1) as g:
        g.set_system(s.L_mo, s.h_mo, s.eps)
        g.set_initial_amplitudes_guess()
        g.set_term_timing(True)
        g.construct_omega()
        g.construct_omega()
        g.jacobian_transformation(g.get_amplitudes())
        log = g.term_timings()
        g.set_term_timing(False)
        for label in ("Construct CCSD Omega", "omega ccsd a2", "omega ccsd c2 and d2", "omega ccsd b2",
                      "omega ccsd e2", "omega doubles a1", "Construct u_aibj", "Jacobian CCSD transformation"):
            assert label in log, (label, sorted(log))
            assert log[label]["calls"] >= 1 and log[label]["ms"] > 0.0
        assert log["Construct CCSD Omega"]["calls"] == 2
        # the residual's terms are parts of it
        parts = sum(log[k]["ms"] for k in ("omega ccsd a2", "omega ccsd c2 and d2", "omega ccsd b2"))
        assert parts <= log["Construct CCSD Omega"]["ms"] + log["Jacobian CCSD transformation"]["ms"]
        g.construct_omega()
        assert g.term_timings() == log      # logging off: nothing new recorded
