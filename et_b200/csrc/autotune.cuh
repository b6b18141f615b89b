// Measured routes for the GEMMs of the mixed-precision path.
#pragma once

#include <cuda_bf16.h>

#include <functional>
#include <string>
#include <vector>

#include "common.cuh"

namespace ccsd {

// Route of one GEMM shape: 0 = cuBLAS DGEMM in FP64, s >= 1 = split-bf16 tensor cores with s K-splits.
// Shapes are keyed by kind, transposes, plane count, K-chunk and m, n, k rounded up to four steps per
// octave, so neighbouring sizes (the trial-vector counts of a Davidson block) share a measurement.
std::string tune_key(char kind, int64_t m, int64_t n, int64_t k, bool tA, bool tB, const Exec &ex);

// Stored route of a key, or -1 if that shape has not been timed in this process (nor loaded from the
// file named by CCSD_GPU_TUNE_FILE).
int tune_lookup(const std::string &key);

// Times every route of `routes` with run(route) on ex.stream (which must write only scratch memory),
// stores and returns the fastest.  Returns -1 without timing while ex.stream is being captured or
// while another thread is timing (the caller then uses its fixed rule for this call).
int tune_measure(Exec &ex, const std::string &key, const std::vector<int> &routes,
                 const std::function<void(int)> &run);

// Number of routes timed and stored by this process (for tests and reports).
int64_t tune_entries();

// tc_gemm_f64 on pre-split operands with its K-split count from the tuner when ex.autotune is set
// (`fixed` otherwise: 0 = wave rule, s >= 1 = that count).
void tc_gemm_f64_tuned(Exec &ex, const __nv_bfloat16 *A, int64_t Mp, const __nv_bfloat16 *B, int64_t Np, int64_t Kp,
                       int64_t m, int64_t n, int64_t k_true, double alpha, double beta, double *C, int64_t ldc,
                       int fixed);

}  // namespace ccsd
