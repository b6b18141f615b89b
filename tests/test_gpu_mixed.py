"""Split-BF16 tcgen05 GEMM and the mixed-precision Omega against FP64 references."""

import numpy as np
import pytest

from et_b200.synthetic import make_system
from oracle import ccsd as oc

pytestmark = pytest.mark.gpu

# bf16 hi+lo keeps ~16 significant bits per operand; the dropped lo*lo product and the FP32
# accumulation leave a relative error of order 1e-5 per dot product.
GEMM_RTOL = 1e-4
# three planes keep ~24 bits of each operand; what remains is the FP32 accumulation in TMEM, so
# the three-plane mode is much tighter than two planes for short K and about as tight for long K.
GEMM_RTOL_X6 = 1e-5


@pytest.fixture(scope="module")
def ctx():
    from et_b200 import CCSD
    c = CCSD(2, 3, 4)
    yield c
    c.close()


@pytest.mark.parametrize("m,n,k", [(128, 256, 64), (200, 300, 100), (1, 1, 16), (129, 257, 65),
                                   (640, 512, 1200), (300, 1000, 777),
                                   (200, 300, 20000), (320, 320, 41000)])   # the last two run split-K
@pytest.mark.parametrize("tA,tB", [(False, False), (True, False), (False, True), (True, True)])
def test_mixed_gemm_matches_fp64(ctx, m, n, k, tA, tB):
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    A = rng.standard_normal((k, m) if tA else (m, k))
    B = rng.standard_normal((n, k) if tB else (k, n))
    C0 = rng.standard_normal((m, n))
    ref = 0.7 * ((A.T if tA else A) @ (B.T if tB else B)) - 0.3 * C0
    out = ctx.selftest_gemm(A, B, C0, alpha=0.7, beta=-0.3, transA=tA, transB=tB, mixed=True)
    scale = np.abs(A).max() * np.abs(B).max() * np.sqrt(k)
    assert np.abs(out - ref).max() <= GEMM_RTOL * scale


@pytest.mark.parametrize("m,n,k", [(128, 128, 64), (129, 257, 65), (256, 384, 192), (640, 512, 1200),
                                   (300, 1000, 777), (200, 300, 20000)])
@pytest.mark.parametrize("tA,tB", [(False, False), (True, True)])
def test_mixed6_gemm_matches_fp64(ctx, m, n, k, tA, tB):
    """Three-plane mode (N tile 128): within the bound on every shape, tighter for short K."""
    rng = np.random.default_rng(m * 5 + n * 11 + k)
    A = rng.standard_normal((k, m) if tA else (m, k))
    B = rng.standard_normal((n, k) if tB else (k, n))
    C0 = rng.standard_normal((m, n))
    ref = 0.7 * ((A.T if tA else A) @ (B.T if tB else B)) - 0.3 * C0
    out6 = ctx.selftest_gemm(A, B, C0, alpha=0.7, beta=-0.3, transA=tA, transB=tB, mixed=2)
    out3 = ctx.selftest_gemm(A, B, C0, alpha=0.7, beta=-0.3, transA=tA, transB=tB, mixed=1)
    scale = np.abs(A).max() * np.abs(B).max() * np.sqrt(k)
    err6, err3 = np.abs(out6 - ref).max(), np.abs(out3 - ref).max()
    assert err6 <= GEMM_RTOL_X6 * scale
    if k <= 128:                     # accumulation error takes over from K ~ 200 on
        assert err6 < 0.3 * err3


def test_fp64_gemm_path(ctx):
    rng = np.random.default_rng(3)
    A = rng.standard_normal((70, 50))
    B = rng.standard_normal((50, 90))
    out = ctx.selftest_gemm(A, B, mixed=False)
    assert np.abs(out - A @ B).max() < 1e-12


def test_mixed_gemm_repeatable(ctx):
    """Two calls in a row give bitwise identical results (no state leaks between launches)."""
    rng = np.random.default_rng(5)
    A = rng.standard_normal((300, 200))
    B = rng.standard_normal((200, 400))
    a = ctx.selftest_gemm(A, B, mixed=True)
    b = ctx.selftest_gemm(A, B, mixed=True)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("dims", [(4, 16, 40), (8, 40, 100)])
@pytest.mark.parametrize("start", ["random", "mp2"])
def test_mixed_omega_close_to_oracle(dims, start):
    """Mixed Omega vs the FP64 oracle.  Near the MP2 point Omega is a small difference of large
    terms (g_aibj against the Fock-denominator terms), so the error is measured against the size
    of those terms rather than against |Omega|."""
    from et_b200 import CCSD, MIXED
    n_o, n_v, n_J = dims
    s = make_system(n_o, n_v, n_J, seed=9)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    if start == "mp2":
        ref.mp2_start()
    else:
        ref.set_amplitudes(0.05 * np.random.default_rng(4).standard_normal(ref.n_amp))
    gpu = CCSD(n_o, n_v, n_J, precision=MIXED, mixed_min_flops=1)
    gpu.set_system(s.L_mo, s.h_mo, s.eps)
    gpu.set_amplitudes(ref.get_amplitudes())
    om = gpu.construct_omega()
    om_ref = ref.omega()
    ladder = oc.omega_ccsd_a2_dense(oc.squareup(ref.t2, ref.n_v, ref.n_o), ref.L_t1, ref.n_o)
    L_vo = ref.L_t1[:, ref.n_o:, :ref.n_o]
    g_vovo = oc.packin(oc.eri(L_vo, L_vo), ref.n_v, ref.n_o)
    scale = max(np.linalg.norm(om_ref), np.linalg.norm(ladder), np.linalg.norm(g_vovo))
    assert np.linalg.norm(om - om_ref) <= 1e-4 * scale
    gpu.close()


def test_mixed_solver_refines_to_fp64_energy():
    """Mixed iterations followed by FP64 refinement land on the FP64 energy (|dE| <= 1e-8 Eh)."""
    from et_b200 import CCSD, FP64, MIXED
    n_o, n_v, n_J = 6, 40, 120
    s = make_system(n_o, n_v, n_J, seed=21)
    res = {}
    for prec in (FP64, MIXED):
        gpu = CCSD(n_o, n_v, n_J, precision=prec, mixed_min_flops=1)
        gpu.set_system(s.L_mo, s.h_mo, s.eps)
        gpu.set_initial_amplitudes_guess()
        e, it, hist, rc = gpu.solve_ground_state(omega_threshold=1e-9, energy_threshold=1e-11,
                                                 refine_threshold=1e-5, raise_on_failure=False)
        assert rc == 0, f"precision {prec}: {it} iterations, |Omega| history {hist[:, 1].tolist()}"
        res[prec] = e
        gpu.close()
    assert abs(res[MIXED] - res[FP64]) <= 1e-8


@pytest.mark.parametrize("batch", [1, 3, 16])
def test_mixed_ladder_batching(batch):
    """Tensor-core ladder: any a-batch of the pair-integral GEMM gives the same Omega."""
    from et_b200 import CCSD, MIXED
    n_o, n_v, n_J = 5, 19, 33
    s = make_system(n_o, n_v, n_J, seed=13)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    ref.set_amplitudes(0.05 * np.random.default_rng(2).standard_normal(ref.n_amp))
    gpu = CCSD(n_o, n_v, n_J, precision=MIXED, mixed_min_flops=1, ladder_batch=batch)
    gpu.set_system(s.L_mo, s.h_mo, s.eps)
    gpu.set_amplitudes(ref.get_amplitudes())
    om, om_ref = gpu.construct_omega(), ref.omega()
    assert np.linalg.norm(om - om_ref) <= 1e-4 * np.linalg.norm(om_ref)
    gpu.close()


def test_chunked_accumulation_beats_whole_k_accumulation():
    """Long K (no split-K: 16 x 10 output tiles): the tensor cores' FP32 accumulation truncates a
    little at every step, so summing 4096-wide chunks in FP64 removes most of the drift.  Seen
    clearly on non-negative operands, where the truncation adds up to a one-sided bias."""
    from et_b200 import CCSD
    m, n, k = 2048, 2560, 32768
    rng = np.random.default_rng(8)
    A = np.abs(rng.standard_normal((m, k)))
    B = np.abs(rng.standard_normal((k, n)))
    ref = A @ B
    rel = {}
    for chunk in (0, -1):            # 0: the default 4096-wide chunks; -1: one accumulator for all of K
        with CCSD(2, 3, 4, mixed_k_chunk=chunk) as c:
            out = c.selftest_gemm(A, B, mixed=True)
        rel[chunk] = (out - ref) / ref
    bias_chunked, bias_whole = abs(rel[0].mean()), abs(rel[-1].mean())
    assert np.abs(rel[0]).max() < 1e-4
    assert bias_chunked < 0.5 * bias_whole, (bias_chunked, bias_whole)



def test_mixed_jacobian_and_transpose_close_to_fp64():
    """Tangent and adjoint contractions through the tensor cores (permuted operands and outputs are
    read and written in place) against the FP64 transformations."""
    from et_b200 import CCSD, FP64, MIXED
    n_o, n_v, n_J = 6, 40, 90
    s = make_system(n_o, n_v, n_J, seed=31)
    rng = np.random.default_rng(7)
    out = {}
    for prec in (FP64, MIXED):
        with CCSD(n_o, n_v, n_J, precision=prec, mixed_min_flops=1) as g:
            g.set_system(s.L_mo, s.h_mo, s.eps)
            g.set_initial_amplitudes_guess()
            C = np.random.default_rng(3).standard_normal((g.n_amp, 3))
            out[prec] = (g.jacobian_transformation(C), g.jacobian_transpose_transformation(C))
    for k in range(2):
        ref, mix = out[FP64][k], out[MIXED][k]
        assert np.linalg.norm(mix - ref) <= 1e-4 * np.linalg.norm(ref)


@pytest.mark.parametrize("dims", [(5, 19, 33), (6, 32, 70)])
def test_mixed_singles_jacobian_with_t1_matches_fp64(dims):
    """Singles trial vectors at amplitudes with sizeable t1: the ladder's t1 tangent takes Y from the
    resident untransformed ovvv integrals plus the correction -sum_l t_bl Q_kilj for the
    T1-transformed vv block.  The mixed result must agree with FP64 far more closely than the size
    of that ladder term (a missing or wrong correction shows up at ~20 % of it)."""
    from et_b200 import CCSD, FP64, MIXED
    n_o, n_v, n_J = dims
    s = make_system(n_o, n_v, n_J, seed=41)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    amp = 0.05 * np.random.default_rng(5).standard_normal(ref.n_amp)
    amp[: ref.n_t1] *= 3.0
    ref.set_amplitudes(amp)
    C = np.zeros((ref.n_amp, 2))
    C[: ref.n_t1] = np.random.default_rng(6).standard_normal((ref.n_t1, 2))
    out = {}
    for prec in (FP64, MIXED):
        with CCSD(n_o, n_v, n_J, precision=prec, mixed_min_flops=1) as g:
            g.set_system(s.L_mo, s.h_mo, s.eps)
            g.set_amplitudes(amp)
            out[prec] = (g.jacobian_transformation(C), g.jacobian_transpose_transformation(C))
    # the ladder's t1 tangent, -sum_k c_ak Y_kibj with Y_kibj = sum_cd g_kc~bd t_cidj
    o = n_o
    Lt = ref.L_t1
    g_ovvv = np.einsum("Jkc,Jbd->kcbd", Lt[:, :o, o:], Lt[:, o:, o:])
    tf = oc.squareup(ref.t2, ref.n_v, ref.n_o)
    Y = np.einsum("kcbd,cidj->kibj", g_ovvv, tf)
    for k in range(2):
        c1 = C[: ref.n_t1, k].reshape(n_v, n_o, order="F")
        ladder_t1 = np.linalg.norm(np.einsum("ak,kibj->aibj", c1, Y))
        for which in range(2):
            r64, rmx = out[FP64][which][:, k], out[MIXED][which][:, k]
            err = np.linalg.norm(rmx - r64)
            assert err <= 1e-4 * np.linalg.norm(r64)
            if which == 0:
                assert err <= 1e-3 * ladder_t1, (err, ladder_t1)


@pytest.mark.parametrize("dims", [(5, 19, 33), (6, 40, 90)])
def test_streamed_ladder_equals_resident(dims):
    """A pair-integral budget below the resident size forms the split-bf16 ladder integrals block by
    block in every call (eT's (a, b) batching).  With one K split (the fixed GEMM rule) every output
    element is the same dot product, so Omega, A c and A^T b equal the resident form's bit for bit,
    for one a per block (budget 1 byte) and for blocks of several a."""
    from et_b200 import CCSD, MIXED
    n_o, n_v, n_J = dims
    s = make_system(n_o, n_v, n_J, seed=23)
    rng = np.random.default_rng(4)
    row_bytes = 2 * 2 * ((n_v * n_v + 63) // 64 * 64)
    res = {}
    for budget in (0, 1, (3 * n_v + 128) * row_bytes):
        with CCSD(n_o, n_v, n_J, precision=MIXED, mixed_min_flops=1, ladder_pair_budget=budget) as g:
            g.set_system(s.L_mo, s.h_mo, s.eps)
            amp = 0.05 * np.random.default_rng(4).standard_normal(g.n_amp)
            g.set_amplitudes(amp)
            C = np.random.default_rng(5).standard_normal((g.n_amp, 2))
            res[budget] = (g.construct_omega(), g.jacobian_transformation(C), g.jacobian_transpose_transformation(C))
    for budget in list(res)[1:]:
        for x, y in zip(res[0], res[budget]):
            assert np.array_equal(x, y), budget


def test_gathered_operands_equal_reordered_copies():
    """An operand whose indices are not two contiguous groups (a 4-index block contracted over a
    scattered pair of its indices) is split into bf16 planes straight from its own layout once its
    product's route is known to be the tensor cores; before that (the first call of a shape, timed by
    the autotuner) it goes through a reordered FP64 copy.  Both give the same planes, so the second
    residual equals the first bit for bit, and every later call launches the same kernels."""
    from et_b200 import CCSD, MIXED
    n_o, n_v, n_J = 7, 45, 110                     # shapes no other test tunes
    s = make_system(n_o, n_v, n_J, seed=31)
    with CCSD(n_o, n_v, n_J, precision=MIXED, mixed_min_flops=1, autotune=1) as g:
        g.set_system(s.L_mo, s.h_mo, s.eps)
        g.set_amplitudes(0.05 * np.random.default_rng(6).standard_normal(g.n_amp))
        first = g.construct_omega()
        n0, _ = g.stats()
        g.set_profiling(True)
        second = g.construct_omega()
        n1, _ = g.stats()
        third = g.construct_omega()
        n2, _ = g.stats()
        tc_launches, _, _ = g.gemm_profile()
        g.set_profiling(False)
    assert tc_launches > 0
    assert np.array_equal(first, second) and np.array_equal(second, third)
    assert n2 - n1 == n1 - n0


def test_cta_pair_gemm_matches_fp64():
    """The two-plane GEMM on CTA pairs (cta_group::2, M = 256 per pair, CCSD_GPU_PAIR_GEMM=1, read once
    per process) in a fresh process: the same tolerance against FP64 as the single-CTA kernel, with
    transposes, a K split and row counts that leave the second CTA of the last pair without rows."""
    import os
    import subprocess
    import sys
    code = r"""
import numpy as np
from et_b200 import CCSD
rng = np.random.default_rng(7)
with CCSD(2, 3, 4) as c:
    for (m, n, k, tA, tB) in [(256, 256, 64, False, False), (300, 1000, 777, True, False),
                              (640, 512, 1200, False, True), (384, 300, 20000, True, True)]:
        A = rng.standard_normal((k, m) if tA else (m, k))
        B = rng.standard_normal((n, k) if tB else (k, n))
        ref = (A.T if tA else A) @ (B.T if tB else B)
        out = c.selftest_gemm(A, B, transA=tA, transB=tB, mixed=1)
        scale = np.abs(A).max() * np.abs(B).max() * np.sqrt(k)
        err = np.abs(out - ref).max() / scale
        assert err < 1e-4, (m, n, k, tA, tB, err)
print("ok")
"""
    env = dict(os.environ, CCSD_GPU_PAIR_GEMM="1")
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    r = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "ok" in r.stdout, r.stderr[-2000:]
