"""The FP64-accurate int8 digit GEMM (tcgen05 kind::i8, et_b200/csrc/ozaki_gemm.cu): bit for bit
against its CPU emulation (tests/ozaki_reference.py), against FP64 with alpha/beta and transposes,
and inside the residual and the mixed-precision solver's FP64 evaluations."""

import numpy as np
import pytest

import ozaki_reference as oz
from et_b200.synthetic import make_system
from oracle import ccsd as oc

pytestmark = pytest.mark.gpu

SHAPES = [(128, 128, 64), (129, 257, 65), (1, 1, 16), (300, 1000, 777), (256, 384, 16448), (640, 520, 20000)]


@pytest.fixture(scope="module")
def ctx():
    from et_b200 import CCSD
    c = CCSD(2, 3, 4)
    yield c
    c.close()


@pytest.mark.parametrize("m,n,k", SHAPES)
@pytest.mark.parametrize("digits", [7, 5, 4])
def test_digit_gemm_equals_emulation_bitwise(ctx, m, n, k, digits):
    """alpha = 1, beta = 0: exact integer digit products and the same FP64 sums in the same order."""
    rng = np.random.default_rng(m + 3 * n + 7 * k + digits)
    A = rng.standard_normal((m, k)) * np.exp2(rng.integers(-30, 30, size=(m, 1)))
    B = rng.standard_normal((k, n))
    if m > 3:
        A[2] = 0.0                                   # an all-zero row
    out = ctx.selftest_gemm(A, B, mixed=digits)
    assert np.array_equal(out, oz.ozaki_gemm(A, B, digits))


def test_digit_gemm_in_k_slabs_equals_one_launch(ctx, monkeypatch):
    """Operands whose digit planes exceed the slab budget are converted and multiplied in K slabs of
    whole chunks; the result is bit for bit that of one launch over all K."""
    rng = np.random.default_rng(12)
    A = rng.standard_normal((300, 40000))
    B = rng.standard_normal((40000, 200))
    whole = ctx.selftest_gemm(A, B, mixed=7)
    monkeypatch.setenv("CCSD_GPU_DIGIT_SLAB_MB", "1")          # one 16384-wide chunk per slab
    sliced = ctx.selftest_gemm(A, B, mixed=7)
    assert np.array_equal(whole, sliced)
    assert np.array_equal(whole, oz.ozaki_gemm(A, B, 7))


@pytest.mark.parametrize("m,n,k", [(129, 257, 65), (300, 1000, 777), (640, 520, 20000)])
@pytest.mark.parametrize("tA,tB", [(False, False), (True, False), (False, True), (True, True)])
def test_digit_gemm_matches_fp64(ctx, m, n, k, tA, tB):
    rng = np.random.default_rng(m * 5 + n * 11 + k)
    A = rng.standard_normal((k, m) if tA else (m, k))
    B = rng.standard_normal((n, k) if tB else (k, n))
    C0 = rng.standard_normal((m, n))
    ref = 0.7 * ((A.T if tA else A) @ (B.T if tB else B)) - 0.3 * C0
    out = ctx.selftest_gemm(A, B, C0, alpha=0.7, beta=-0.3, transA=tA, transB=tB, mixed=7)
    scale = np.abs(A).max() * np.abs(B).max() * np.sqrt(k)
    assert np.abs(out - ref).max() <= 5e-13 * scale


def test_fp64_residual_with_digit_products_matches_dgemm():
    """Every product of the FP64 residual on the int8 tensor cores (min_flops = 1): within 1e-12
    of the size of its terms of the DGEMM residual, and of the oracle."""
    from et_b200 import CCSD
    n_o, n_v, n_J = 6, 40, 100
    s = make_system(n_o, n_v, n_J, seed=19)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    ref.mp2_start()
    amp = ref.get_amplitudes() * (1.0 + 0.1 * np.random.default_rng(2).standard_normal(ref.n_amp))
    ref.set_amplitudes(amp)
    om_ref = ref.omega()
    L_vo = ref.L_t1[:, n_o:, :n_o]
    scale = max(np.abs(om_ref).max(), np.abs(oc.eri(L_vo, L_vo)).max())
    with CCSD(n_o, n_v, n_J) as g:
        g.set_system(s.L_mo, s.h_mo, s.eps)
        g.set_amplitudes(amp)
        om_dgemm = g.construct_omega()
        g.set_fp64_digits(7, min_flops=1)
        g.set_profiling(True)
        om_digits = g.construct_omega()
        launches, ms, ops = g.digit_gemm_profile()
        g.set_profiling(False)
        g.set_fp64_digits(0)
        assert np.array_equal(g.construct_omega(), om_dgemm)
    assert launches > 10 and ops > 0
    assert np.abs(om_digits - om_dgemm).max() <= 1e-12 * scale
    assert np.abs(om_digits - om_ref).max() <= 1e-12 * scale


def test_mixed_solver_with_digit_refreshes_reaches_fp64_energy():
    """Mixed iterations with FP64-accurate refreshes on the int8 tensor cores land on the DGEMM FP64
    energy (|dE| <= 1e-8 Eh, the benchmark's target), as the DGEMM refreshes do."""
    from et_b200 import CCSD, FP64, MIXED
    n_o, n_v, n_J = 6, 40, 120
    s = make_system(n_o, n_v, n_J, seed=21)
    res = {}
    for name, prec, digits in (("fp64", FP64, -1), ("mixed_digits", MIXED, 7)):
        with CCSD(n_o, n_v, n_J, precision=prec, mixed_min_flops=1) as g:
            g.set_system(s.L_mo, s.h_mo, s.eps)
            g.set_fp64_digits(7 if digits > 0 else 0, min_flops=1)
            g.set_initial_amplitudes_guess()
            e, it, hist, rc = g.solve_ground_state(omega_threshold=1e-9, energy_threshold=1e-11,
                                                   refine_threshold=1e-5, refresh_digits=digits,
                                                   raise_on_failure=False)
            assert rc == 0, (name, it, hist[:, 1].tolist())
            res[name] = e
    assert abs(res["mixed_digits"] - res["fp64"]) <= 1e-8
