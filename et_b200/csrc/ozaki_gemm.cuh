// FP64-accurate GEMM on the int8 tensor cores (tcgen05 kind::i8, Ozaki's error-free digit slicing).
#pragma once

#include "common.cuh"

namespace ccsd {

// C (m x n, col-major, ldc) = alpha op(A) op(B) + beta C with FP64 operands cut into `digits`
// 7-bit int8 digits per row of op(A) / column of op(B) (power-of-two scaled), the digit products
// of weight >= 2^(-7(digits+1)) summed exactly in int32 on the tensor cores and in FP64 by the
// epilogue.  digits = 7: ~1e-14 of the largest output (FP64 DGEMM: ~1e-16).  Deterministic.
// Digit planes of one operand for the whole K, kept by the caller for an operand that takes part in
// many products unchanged (the resident FP64 integrals of the refreshes): int exponents of its rows,
// then int8 planes [digits][Rp][Kp] (rows padded to 128, K to 64).
struct OzPlanes {
    DBuf buf;
    int64_t rows = 0, k = 0, Rp = 0, Kp = 0;
    int digits = 0;
    size_t exp_bytes = 0;
    int8_t *digits_base() const { return reinterpret_cast<int8_t *>(buf.as<uint8_t>() + exp_bytes); }
};
// rows of op(X) (X[r + ldx kk] for trans = false, X[kk + ldx r] for true) cut into `digits` digits
void ozaki_prepare(Exec &ex, bool trans, int64_t rows, int64_t k, const double *X, int64_t ldx, int digits,
                   OzPlanes &out);

// pa / pb: prepared digit planes of op(A) / op(B) (same rows, K and digits); the raw operand is then
// not read
void ozaki_gemm(Exec &ex, bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha,
                const double *A, int64_t lda, const double *B, int64_t ldb, double beta, double *C, int64_t ldc,
                int digits = 7, const OzPlanes *pa = nullptr, const OzPlanes *pb = nullptr);

// int8 digit products one ozaki_gemm issues per output element and K index
int ozaki_products(int digits);

}  // namespace ccsd
