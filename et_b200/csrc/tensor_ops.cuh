// Tensor primitives of libccsd_gpu: strided permute/add, GEMM-based contractions, packing.
#pragma once

#include "common.cuh"

namespace ccsd {

// out = alpha * permute(in) + beta * out.  `in` and `out` describe the same logical
// dimensions (n[k] equal), with their own strides.
void permute_add(Exec &ex, double alpha, const TV &in, double beta, const TV &out);

// Einstein-summation contraction of two operands through one GEMM:
//   C[lc] = alpha * sum_{k} A[la] B[lb] + beta * C[lc]
// spec "la,lb->lc"; every label of A and B appears in exactly two of the three views.
void contract(Exec &ex, const char *spec, double alpha, const TV &A, const TV &B, double beta,
              const TV &C);

// C (m x n, col-major, ldc) = alpha op(A) op(B) + beta C.  FP64 DGEMM, or the tcgen05
// split-BF16 GEMM when ex.prec == MIXED and 2mnk >= ex.mixed_min_flops.
void gemm(Exec &ex, bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha,
          const double *A, int64_t lda, const double *B, int64_t ldb, double beta, double *C,
          int64_t ldc, bool allow_mixed = true);

// C_z = alpha op(A_z) op(B_z) + beta C_z for z < batch, operand z at base + z * stride (FP64
// DGEMM, strided batch): a product whose output index sits between two batch indices
void gemm_batched_f64(Exec &ex, bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha,
                      const double *A, int64_t lda, int64_t strideA, const double *B, int64_t ldb, int64_t strideB,
                      double beta, double *C, int64_t ldc, int64_t strideC, int64_t batch);

// packed doubles <-> full symmetric (v,o,v,o)
void squareup(Exec &ex, const double *packed, double *full, int64_t nov);
// packed += alpha * full(M,m) * (1/2 if M == m) over M >= m (eT's scale_diagonal(1/2) + packin);
// reads the symmetric counterpart full(m, M) for coalescing, so `full` must be symmetric.
void pack_half_diag_add(Exec &ex, double alpha, const double *full, double *packed, int64_t nov);

// reductions (deterministic two-pass)
void dot(Exec &ex, const double *x, const double *y, int64_t n, double *d_result);
void multi_dot(Exec &ex, const double *x, const double *const *ys, int nys, int64_t n, double *d_results);

void fill(Exec &ex, double *p, int64_t n, double value);
void axpby(Exec &ex, int64_t n, double alpha, const double *x, double beta, double *y);

}  // namespace ccsd
