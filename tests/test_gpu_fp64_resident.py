"""FP64 residual from resident integrals of the untransformed Cholesky vectors (the +/- ladder
integrals of all pairs and the ovvv block, plus o^2 v^3 corrections for the T1 transformation)
against the oracle and against eT's per-call T1-transformed integrals."""

import numpy as np
import pytest

from et_b200.synthetic import make_system
from oracle import ccsd as oc

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dims", [(2, 5, 9), (4, 16, 40), (5, 19, 33), (8, 40, 100)])
def test_resident_fp64_omega_matches_oracle_and_per_call_path(dims):
    from et_b200 import CCSD
    n_o, n_v, n_J = dims
    s = make_system(n_o, n_v, n_J, seed=17)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    amp = 0.05 * np.random.default_rng(3).standard_normal(ref.n_amp)
    amp[: ref.n_t1] *= 3.0
    ref.set_amplitudes(amp)
    om_ref = ref.omega()
    out = {}
    for resident in (True, False):
        with CCSD(n_o, n_v, n_J) as g:
            g.set_fp64_integrals(resident)
            g.set_system(s.L_mo, s.h_mo, s.eps)
            g.set_amplitudes(amp)
            out[resident] = g.construct_omega()
    scale = max(1.0, np.abs(om_ref).max())
    assert np.abs(out[True] - om_ref).max() <= 1e-12 * scale
    assert np.abs(out[True] - out[False]).max() <= 1e-12 * scale


def test_resident_fp64_jacobian_with_t1_matches_oracle():
    """The Jacobian's t1 terms take Y from the resident ovvv block plus the T1 correction."""
    from et_b200 import CCSD
    n_o, n_v, n_J = 3, 8, 20
    s = make_system(n_o, n_v, n_J, seed=23)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    amp = 0.1 * np.random.default_rng(4).standard_normal(ref.n_amp)
    ref.set_amplitudes(amp)
    A = ref.jacobian_matrix()
    C = np.random.default_rng(5).standard_normal((ref.n_amp, 3))
    with CCSD(n_o, n_v, n_J) as g:
        g.set_system(s.L_mo, s.h_mo, s.eps)
        g.set_amplitudes(amp)
        R = g.jacobian_transformation(C)
        S = g.jacobian_transpose_transformation(C)
    assert np.abs(R - A @ C).max() <= 1e-11 * max(1.0, np.abs(A).max())
    assert np.abs(S - A.T @ C).max() <= 1e-11 * max(1.0, np.abs(A).max())


def test_resident_fp64_integrals_follow_new_cholesky_vectors():
    from et_b200 import CCSD
    n_o, n_v, n_J = 4, 16, 40
    s = make_system(n_o, n_v, n_J, seed=29)
    L2 = s.L_mo * 0.97
    ref = oc.CCSDSystem(L2, s.h_mo, s.eps, s.n_o)
    amp = 0.05 * np.random.default_rng(6).standard_normal(ref.n_amp)
    ref.set_amplitudes(amp)
    with CCSD(n_o, n_v, n_J) as g:
        g.set_system(s.L_mo, s.h_mo, s.eps)
        g.set_amplitudes(amp)
        g.construct_omega()                # integrals of the first vectors
        g.set_cholesky_mo(L2)
        g.set_amplitudes(amp)
        om = g.construct_omega()
    assert np.abs(om - ref.omega()).max() <= 1e-12 * max(1.0, np.abs(ref.omega()).max())
