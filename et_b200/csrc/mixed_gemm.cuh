// Split-BF16 ("bf16x3") GEMM on the sm_100a tensor cores (tcgen05 + TMEM + TMA).
#pragma once

#include <cuda_bf16.h>

#include <vector>

#include "common.cuh"

namespace ccsd {

// C (m x n, col-major, ldc) = alpha op(A) op(B) + beta C with FP64 operands split into
// bf16 hi + lo parts; the three products hi*hi + hi*lo + lo*hi accumulate in FP32.
// splits: K-split count (<= 0: tc_default_splits).
void mixed_gemm(Exec &ex, bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha,
                const double *A, int64_t lda, const double *B, int64_t ldb, double beta, double *C, int64_t ldc,
                int splits = -1);

// FP64 operand of the tensor-core GEMM as a strided gather: element (r, k) at p[roff(r) + koff(k)],
// roff(r) = sum_d digit_d(r) * rs[d] with the digits of r over the extents rn[0..nr) (first
// fastest), koff(k) likewise over kn/ks.  A tensor whose row or K indices span several dimensions
// (a 4-index amplitude or integral block in any index order) is split straight into bf16 planes.
struct SplitView {
    const double *p;
    int nr, nk;
    long long rn[4], rs[4], kn[4], ks[4];
};
SplitView matrix_view(const double *p, int64_t rows, int64_t sr, int64_t K, int64_t sk);

// C (m x n, col-major, ldc) = alpha A B^T + beta C for operands given as views: A's rows are the m
// output rows, B's rows the n output columns, both with the same k contraction indices.
void mixed_gemm_views(Exec &ex, const SplitView &A, const SplitView &B, int64_t m, int64_t n, int64_t k, double alpha,
                      double beta, double *C, int64_t ldc, int splits = -1);

// Routes (the `splits` argument of the GEMMs below and of mixed_gemm): s in 1..99 runs the
// single-CTA kernel with s K splits, PAIR_ROUTE + s the CTA-pair kernel (cta_group::2, 256 x 256
// tiles) with s K splits; 0 or less takes the fixed rule's count.
constexpr int PAIR_ROUTE = 100;

// K-split count of the fixed rule: split only when the output tiles cannot fill the SMs.
int tc_default_splits(int64_t m, int64_t n, int64_t k, int planes);
// K-split counts worth timing for an m x n x k product: 1, the fixed rule's count, and counts whose
// tile units fill whole waves of the persistent grid; for products of at least 256 rows the same
// counts again as CTA-pair routes.
std::vector<int> tc_split_candidates(int64_t m, int64_t n, int64_t k, int planes);

// Row / K padding of pre-split operands (A rows to 128, B rows to 256, K to 64).
int64_t tc_pad_rows_a(int64_t m);
int64_t tc_pad_rows_b(int64_t n);
int64_t tc_pad_k(int64_t k);

// FP64 strided view (element (r, k) at src[r*sr + k*sk]) -> bf16 hi/lo planes [2][Rp][Kp], zero padded.
void split_rows(Exec &ex, const double *src, int64_t sr, int64_t sk, int64_t R, int64_t K, int64_t Rp, int64_t Kp,
                __nv_bfloat16 *out);

// Tensor-core GEMM on pre-split operands A [2][Mp][Kp], B [2][Np][Kp]:
// C (m x n, col-major, FP64) = alpha A B^T + beta C.  splits > 1 divides K into that many
// deterministic partial products summed afterwards; 0 chooses the count from the tile waves.
void tc_gemm_f64(Exec &ex, const __nv_bfloat16 *A, int64_t Mp, const __nv_bfloat16 *B, int64_t Np, int64_t Kp,
                 int64_t m, int64_t n, int64_t k_true, double alpha, double beta, double *C, int64_t ldc,
                 int splits = 1);

// ovvv integrals g_kcbd = sum_J L_kc L_bd of the untransformed Cholesky vectors as split bf16:
// Lov holds split rows c + nv*k (K = N_J padded to Kp), Lvv split rows d + nv*b; the result goes
// to out[plane][k + no*b][c + nv*d] (row stride out_ld, plane stride out_rows_pad * out_ld).
void tc_gemm_ovvv(Exec &ex, const __nv_bfloat16 *Lov, int64_t ov_rows, const __nv_bfloat16 *Lvv, int64_t vv_rows,
                  int64_t Kp, int64_t no, int64_t nv, __nv_bfloat16 *out, int64_t out_rows_pad, int64_t out_ld,
                  int64_t k_true);

// The same GEMM with its split scratch in a fixed file-scope device array (no allocation);
// synchronous, throws CCSD_GPU_ETIMEOUT when a bounded wait ran out.
void mixed_gemm_noalloc(bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha, const double *A,
                        int64_t lda, const double *B, int64_t ldb, double beta, double *C, int64_t ldc,
                        cudaStream_t stream);

// Error code that a tensor-core GEMM on ex's error word recorded when a bounded barrier wait ran
// out (0 = none); waits for ex.stream first, and clears the word when reset is set.
int gemm_error(Exec &ex, bool reset);

}  // namespace ccsd
