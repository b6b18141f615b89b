// FP64-accurate GEMM on the int8 tensor cores (tcgen05 kind::i8, Ozaki's error-free digit slicing).
#pragma once

#include "common.cuh"

namespace ccsd {

// C (m x n, col-major, ldc) = alpha op(A) op(B) + beta C with FP64 operands cut into `digits`
// 7-bit int8 digits per row of op(A) / column of op(B) (power-of-two scaled), the digit products
// of weight >= 2^(-7(digits+1)) summed exactly in int32 on the tensor cores and in FP64 by the
// epilogue.  digits = 7: ~1e-14 of the largest output (FP64 DGEMM: ~1e-16).  Deterministic.
void ozaki_gemm(Exec &ex, bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha,
                const double *A, int64_t lda, const double *B, int64_t ldb, double beta, double *C, int64_t ldc,
                int digits = 7);

// int8 digit products one ozaki_gemm issues per output element and K index
int ozaki_products(int digits);

}  // namespace ccsd
