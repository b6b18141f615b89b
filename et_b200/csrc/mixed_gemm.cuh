// Split-BF16 ("bf16x3") GEMM on the sm_100a tensor cores (tcgen05 + TMEM + TMA).
#pragma once

#include "common.cuh"

namespace ccsd {

// C (m x n, col-major, ldc) = alpha op(A) op(B) + beta C with FP64 operands split into
// bf16 hi + lo parts; the three products hi*hi + hi*lo + lo*hi accumulate in FP32.
void mixed_gemm(Exec &ex, bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha,
                const double *A, int64_t lda, const double *B, int64_t ldb, double beta, double *C, int64_t ldc);

// Error code recorded by a tensor-core GEMM whose bounded barrier wait timed out (0 = none).
int mixed_gemm_error_flag(bool reset);

}  // namespace ccsd
