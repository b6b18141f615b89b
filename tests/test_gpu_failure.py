"""Failure path of the tensor-core GEMM, made on purpose without faulting the GPU.

Every barrier wait of split_bf16_gemm_kernel is bounded.  ccsd_gpu_selftest_gemm_stall runs one
GEMM whose TMA producer withholds the loads of its first pipeline stage (a barrier that nothing
completes), so the MMA warp's wait runs out after a short, given number of cycles.  The kernel then
records a code in the calling context's error word, drains the loads it did issue, frees its TMEM
and returns; the host reads the word and reports CCSD_GPU_ETIMEOUT.  The context (and any other
context) must stay usable afterwards.
"""

import numpy as np
import pytest

from et_b200.synthetic import make_system
from oracle import ccsd as oc

pytestmark = pytest.mark.gpu

ETIMEOUT = -9
SHORT_WAIT = 20_000_000      # SM clock cycles: ~10 ms at 1.9 GHz
GEMM_RTOL = 1e-4             # the split-bf16 GEMM tolerance of tests/test_gpu_mixed.py


def _product_ok(ctx, rng):
    A = rng.standard_normal((300, 200))
    B = rng.standard_normal((200, 400))
    out = ctx.selftest_gemm(A, B, mixed=True)
    scale = np.abs(A).max() * np.abs(B).max() * np.sqrt(200)
    return np.abs(out - A @ B).max() <= GEMM_RTOL * scale


def test_stalled_gemm_reports_timeout_and_context_recovers():
    from et_b200 import CCSD
    rng = np.random.default_rng(3)
    with CCSD(2, 3, 4) as ctx, CCSD(2, 3, 4) as other:
        assert ctx.selftest_gemm_stall(256, 512, 320, wait_cycles=SHORT_WAIT) == ETIMEOUT
        assert "timed out" in ctx.lib.ccsd_gpu_last_error(ctx.ctx).decode()
        # the word was read and cleared: normal products on the same context succeed
        assert _product_ok(ctx, rng)
        # the other context's error word was never touched
        assert _product_ok(other, rng)
        # and the failure is reported again, not swallowed, on a second stall
        assert ctx.selftest_gemm_stall(128, 256, 64, wait_cycles=SHORT_WAIT) == ETIMEOUT
        assert _product_ok(ctx, rng)


def test_stall_with_several_tiles_and_k_blocks():
    """Every CTA of a multi-tile grid withholds its first stage; all of them must time out, drain
    and exit (no CTA may leave loads in flight)."""
    from et_b200 import CCSD
    rng = np.random.default_rng(4)
    with CCSD(2, 3, 4) as ctx:
        assert ctx.selftest_gemm_stall(1024, 1024, 1024, wait_cycles=SHORT_WAIT) == ETIMEOUT
        assert _product_ok(ctx, rng)


def test_mixed_residual_after_a_stall_matches_oracle():
    from et_b200 import CCSD, MIXED
    n_o, n_v, n_J = 4, 16, 40
    s = make_system(n_o, n_v, n_J, seed=9)
    ref = oc.CCSDSystem(s.L_mo, s.h_mo, s.eps, s.n_o)
    ref.set_amplitudes(0.05 * np.random.default_rng(4).standard_normal(ref.n_amp))
    with CCSD(n_o, n_v, n_J, precision=MIXED, mixed_min_flops=1) as gpu:
        gpu.set_system(s.L_mo, s.h_mo, s.eps)
        gpu.set_amplitudes(ref.get_amplitudes())
        assert gpu.selftest_gemm_stall(256, 256, 256, wait_cycles=SHORT_WAIT) == ETIMEOUT
        om, om_ref = gpu.construct_omega(), ref.omega()
        assert np.linalg.norm(om - om_ref) <= 1e-4 * np.linalg.norm(om_ref)
