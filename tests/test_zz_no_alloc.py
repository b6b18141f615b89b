"""The allocation-free tensor-core GEMM entry point against the allocating one.

ccsd_gpu_mixed_gemm_noalloc serves callers that cannot allocate device memory when they call in
(a host program that already gave the whole GPU to its own pool, or a path that must avoid the
synchronisation of cudaMalloc/cudaFree).  Its split scratch is a fixed array inside the library,
so the test hands it device buffers it owns and compares the product with the regular entry point
(ccsd_gpu_selftest_gemm, which allocates its scratch) on two calls in a row.  This file is named
to be collected last.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GEMM_RTOL = 1e-4   # the tolerance of the split-bf16 GEMM tests


def _call(lib, A_d, B_d, C_d, m, n, k, alpha, beta, stream):
    return lib.ccsd_gpu_mixed_gemm_noalloc(0, 0, m, n, k, alpha, ctypes.c_void_p(A_d.data_ptr()), m,
                                           ctypes.c_void_p(B_d.data_ptr()), k, beta,
                                           ctypes.c_void_p(C_d.data_ptr()), m, ctypes.c_void_p(stream))


def test_noalloc_gemm_matches_allocating_entry_point_twice():
    import torch
    from et_b200 import CCSD
    from et_b200.ccsd import load_library
    lib = load_library()
    m, n, k = 300, 500, 700
    rng = np.random.default_rng(11)
    A = rng.standard_normal((m, k))
    B = rng.standard_normal((k, n))
    C0 = rng.standard_normal((m, n))
    with CCSD(2, 3, 4) as ctx:
        ref = ctx.selftest_gemm(A, B, C0, alpha=0.5, beta=-1.25, mixed=True)
    dev = torch.device("cuda:0")
    A_d = torch.from_numpy(np.asfortranarray(A).ravel(order="F")).to(dev)
    B_d = torch.from_numpy(np.asfortranarray(B).ravel(order="F")).to(dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    scale = np.abs(A).max() * np.abs(B).max() * np.sqrt(k)
    for _ in range(2):
        C_d = torch.from_numpy(np.asfortranarray(C0).ravel(order="F")).to(dev)
        rc = _call(lib, A_d, B_d, C_d, m, n, k, 0.5, -1.25, stream)
        assert rc == 0, lib.ccsd_gpu_last_error(None)
        out = C_d.cpu().numpy().reshape(m, n, order="F")
        assert np.abs(out - ref).max() <= GEMM_RTOL * scale
        exact = 0.5 * (A @ B) - 1.25 * C0
        assert np.abs(out - exact).max() <= GEMM_RTOL * scale


def test_noalloc_gemm_rejects_sizes_beyond_its_scratch():
    import torch
    from et_b200.ccsd import load_library
    lib = load_library()
    dev = torch.device("cuda:0")
    x = torch.zeros(16, dtype=torch.float64, device=dev)
    m = n = k = 4096          # 2 x (4096 + 4096) x 4096 bf16 > the fixed 8 Mi-element scratch
    rc = lib.ccsd_gpu_mixed_gemm_noalloc(0, 0, m, n, k, 1.0, ctypes.c_void_p(x.data_ptr()), m,
                                         ctypes.c_void_p(x.data_ptr()), k, 0.0, ctypes.c_void_p(x.data_ptr()), m,
                                         ctypes.c_void_p(0))
    assert rc == -1
    assert b"exceeds the fixed scratch" in lib.ccsd_gpu_last_error(None)
