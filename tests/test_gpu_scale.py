"""Parity at the adjoint-check shape o=16, v=128, N_J=432 (t = MP2 guess x (1 + 0.1 N(0,1))).

At this size the tensor-core GEMM runs the regime of the benchmark: the ladder's K is v^2 = 16384
(four 4096-wide chunks summed in FP64), products small enough for split-K, and, with autotuning,
measured routes.  The FP64 device residual and both Jacobian transformations are compared element
by element with the oracle (FP64, numpy; its dense g_vvvv is 2.1 GB here), and the mixed residual
within the split-bf16 tolerance of tests/test_gpu_mixed.py.  The transpose is checked through
<sigma, c> = <b, A c> with A c from the oracle (complex-step, exact to rounding).
"""

import numpy as np
import pytest

from et_b200.synthetic import make_system
from oracle import ccsd as oc

pytestmark = pytest.mark.gpu

DIMS = (16, 128, 432)


@pytest.fixture(scope="module")
def case():
    n_o, n_v, n_J = DIMS
    s = make_system(n_o, n_v, n_J, seed=2026)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o, s.e_hf)
    ref.mp2_start()
    amp = ref.get_amplitudes()
    rng = np.random.default_rng(7)
    amp = amp * (1.0 + 0.1 * rng.standard_normal(amp.size))
    ref.set_amplitudes(amp)
    om_ref = ref.omega()
    c = rng.standard_normal(ref.n_amp)
    b = rng.standard_normal(ref.n_amp)
    Ac_ref = ref.jacobian_transformation(c)
    L_vo = ref.L_t1[:, n_o:, :n_o]
    g_vovo = oc.packin(oc.eri(L_vo, L_vo), n_v, n_o)
    ladder = oc.omega_ccsd_a2_dense(oc.squareup(ref.t2, n_v, n_o), ref.L_t1, n_o)
    return {"s": s, "amp": amp, "om_ref": om_ref, "c": c, "b": b, "Ac_ref": Ac_ref, "energy": ref.energy(),
            "scale_max": max(np.abs(om_ref).max(), np.abs(g_vovo).max()),
            "scale_norm": max(np.linalg.norm(om_ref), np.linalg.norm(g_vovo), np.linalg.norm(ladder))}


def _gpu(case, **kw):
    from et_b200 import CCSD
    s = case["s"]
    g = CCSD(*DIMS, **kw)
    g.set_system(s.L_mo, s.h_mo, s.eps, s.e_hf)
    g.set_amplitudes(case["amp"])
    return g


@pytest.mark.parametrize("resident", [True, False])
def test_fp64_omega_and_energy_at_scale(case, resident):
    """Both FP64 ladder algorithms: resident integrals of the untransformed vectors + T1 corrections,
    and eT's T1-transformed integrals formed per call."""
    with _gpu(case) as g:
        g.set_fp64_integrals(resident)
        om = g.construct_omega()
        assert np.abs(om - case["om_ref"]).max() <= 1e-11 * case["scale_max"]
        assert abs(g.calculate_energy() - case["energy"]) <= 1e-11 * max(1.0, abs(case["energy"]))


def test_fp64_jacobian_and_transpose_at_scale(case):
    with _gpu(case) as g:
        g.prepare_for_jacobian(0)
        rho = g.jacobian_transformation(case["c"])
        Ac = case["Ac_ref"]
        assert np.abs(rho - Ac).max() <= 1e-11 * np.abs(Ac).max()
        sigma = g.jacobian_transpose_transformation(case["b"])
        lhs, rhs = float(sigma @ case["c"]), float(case["b"] @ Ac)
        assert abs(lhs - rhs) <= 1e-11 * np.linalg.norm(sigma) * np.linalg.norm(case["c"])


@pytest.mark.parametrize("autotune", [1, -1])
def test_mixed_omega_at_scale(case, autotune):
    """Every product on the tensor cores (mixed_min_flops = 1) with measured routes (autotune = 1:
    DGEMM or tensor cores, K-split counts) or the fixed rule (autotune = -1)."""
    from et_b200 import MIXED
    with _gpu(case, precision=MIXED, mixed_min_flops=1, autotune=autotune) as g:
        om = g.construct_omega()
        err = np.linalg.norm(om - case["om_ref"])
        assert err <= 1e-4 * case["scale_norm"], (err, case["scale_norm"])
        # the mixed transformation through the tensor cores, on a preparation
        g.prepare_for_jacobian(0)
        rho = g.jacobian_transformation(case["c"])
        assert np.linalg.norm(rho - case["Ac_ref"]) <= 1e-4 * np.linalg.norm(case["Ac_ref"])
