/*
 * ccsd_gpu.h - C ABI of the B200 (sm_100a) CCSD hot path.
 *
 * The entry points replace the bodies of eT's type-bound procedures on
 * class(ccsd) (paths relative to the eT source tree).  eT's Fortran binds
 * them through an ISO_C_BINDING interface block in the style of
 * src/libint/eri_cdef.F90:25-68 (bind(C), value scalars, real(c_double)
 * arrays), one interface per function below.
 *
 * Conventions (identical to eT):
 *  - every array is column-major double precision and owned by the caller;
 *  - integers are int64_t (eT builds with 64-bit default integers,
 *    CMakeLists.txt:38);
 *  - singles are (n_v, n_o) with ai = a + n_v*i; doubles are upper-packed over
 *    (ai, bj), index max(ai,bj)*(max(ai,bj)+1)/2 + min(ai,bj) (0-based form of
 *    src/tools/reordering.F90:4174-4198); an amplitude-like vector is
 *    [singles (n_t1) | packed doubles (n_t2)], n_t1 = n_o*n_v,
 *    n_t2 = n_t1*(n_t1+1)/2;
 *  - Cholesky vectors are L[J, p, q] with J fastest over the full MO range
 *    (occupied first): g_pqrs = sum_J L^J_pq L^J_rs
 *    (src/eri_tool/eri_tool_class.F90:92-163).
 *
 * Every function returns 0 on success or a negative CCSD_GPU_E* status;
 * ccsd_gpu_last_error() returns a message for the last failure on a context.
 * A context owns one CUDA stream; calls on one context must come from one
 * host thread at a time.  Distinct contexts are independent.
 */
#ifndef CCSD_GPU_H
#define CCSD_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CCSD_GPU_OK = 0,
    CCSD_GPU_EINVAL = -1,        /* bad dimensions / arguments */
    CCSD_GPU_ECUDA = -2,         /* CUDA runtime or cuBLAS error */
    CCSD_GPU_ENOMEM = -3,        /* device allocation failed */
    CCSD_GPU_ESTATE = -4,        /* required input not set yet */
    CCSD_GPU_ENOCONV = -5,       /* solver did not converge */
    CCSD_GPU_ENAN = -6,          /* non-finite value detected */
    CCSD_GPU_ESINGULAR = -7,     /* DIIS / reduced-space system singular */
    CCSD_GPU_ENODEV = -8,        /* no sm_100 device available */
    CCSD_GPU_ETIMEOUT = -9       /* a tensor-core GEMM's bounded barrier wait ran out (the GEMM
                                    stopped early; the context stays usable) */
};

/* arithmetic used by the contractions */
enum {
    CCSD_GPU_FP64 = 0,           /* FP64 everywhere (DGEMM on the FP64 tensor pipe) */
    CCSD_GPU_MIXED = 1           /* large contractions as split-BF16 (2 planes, 3 products) tcgen05
                                    GEMMs, FP32 accumulation; everything else FP64 */
};

typedef struct ccsd_gpu_options {
    int32_t device;              /* CUDA ordinal */
    int32_t precision;           /* CCSD_GPU_FP64 or CCSD_GPU_MIXED */
    int64_t ladder_batch;        /* virtual-index batch of the A2 ladder, 0 = automatic */
    int64_t mixed_min_flops;     /* contractions below this many flops stay FP64 (0 = default) */
    int64_t mixed_k_chunk;       /* K elements a tensor-core FP32 accumulator sums before the partial
                                    sum is added in FP64 (0 = default 4096, negative = the whole K) */
    int64_t autotune;            /* MIXED only: route of each GEMM shape (FP64 DGEMM or tensor cores,
                                    K-split count) timed once per process: 1 on, -1 off (fixed flop
                                    threshold and split rule), 0 = on unless mixed_min_flops is given
                                    or the environment sets CCSD_GPU_AUTOTUNE=0 */
    int64_t ladder_pair_budget;  /* MIXED only: bytes the split-bf16 A2 pair integrals of all v(v+1)/2 pairs
                                    may take when kept on the device (0 = half of the free memory);
                                    beyond it they are formed block by block in every call into a buffer
                                    of at most this size (eT's (a, b) batching of omega_ccsd_a2) */
    int64_t reserved[2];
} ccsd_gpu_options;

typedef struct ccsd_gpu_solver_options {
    int32_t max_iterations;      /* diis_cc_gs default 100 (src/solvers/cc/diis_cc_gs_class.F90:139) */
    int32_t diis_dimension;      /* default 8 */
    double omega_threshold;      /* |Omega| convergence threshold */
    double energy_threshold;     /* |dE| convergence threshold (< 0 disables the energy test) */
    double refine_threshold;     /* MIXED only: |Omega| of the first FP64 refresh (default 1e-4) */
    double refine_target;        /* MIXED only: the true residual the refinement aims at; refreshes
                                    that remove drift happen only while the drift exceeds it
                                    (0 = omega_threshold) */
    int32_t refresh_digits;      /* MIXED only: arithmetic of the FP64 evaluations (refreshes and the
                                    FP64 iterations after them): 4..7 = the FP64-accurate int8 digit GEMM
                                    on the tensor cores with that many 7-bit digits per operand for
                                    products of at least 1e10 flops, -1 = cuBLAS DGEMM for every
                                    product, 0 = the default (cuBLAS DGEMM) */
    int32_t reserved[5];
} ccsd_gpu_solver_options;

/* Creation / teardown.  Replaces the wavefunction set-up that allocates t, Omega and the
 * Cholesky storage (src/wavefunctions/ccsd/ccsd_class.F90, src/eri_tool/eri_cholesky_memory_class.F90). */
int  ccsd_gpu_create(int64_t n_o, int64_t n_v, int64_t n_J, const ccsd_gpu_options *opt, void **ctx);
void ccsd_gpu_destroy(void *ctx);
const char *ccsd_gpu_last_error(void *ctx);
int  ccsd_gpu_set_precision(void *ctx, int32_t precision);
/* Run the context's work on a caller-provided stream (a cudaStream_t passed as void*);
 * NULL restores the context's own stream. */
int  ccsd_gpu_set_stream(void *ctx, void *stream);
int  ccsd_gpu_synchronize(void *ctx);

/* MO Cholesky vectors L[J,p,q] over the full MO range (wf%L_mo, set in
 * src/engines/cc/tasks/cholesky_decomposition_task_class.F90:68-138). */
int ccsd_gpu_set_cholesky_mo(void *ctx, const double *L);
/* Same data in eT's four o/v blocks, each (n_J, len_p, len_q)
 * (src/eri_tool/abstract_eri_cholesky_class.F90:290-327). */
int ccsd_gpu_set_cholesky_mo_blocks(void *ctx, const double *L_oo, const double *L_ov,
                                    const double *L_vo, const double *L_vv);
/* MO Cholesky vectors built on the device from the three-index AO integrals of the Cholesky basis,
 * as construct_cholesky_mo_vectors (src/solvers/cholesky/eri_cd_class.F90:3132-3472) does:
 *   L_Jpq = sum_wx C_wp C_xq sum_K (wx|K) [Q^{-T}]_KJ,   S_KL = (K|L) = Q Q^T (Q lower triangular).
 * W_ao: (wx|K) as (n_ao, n_ao, n_J) column-major for the n_J elements K of the Cholesky basis;
 * S: (K|L), n_J x n_J; C: n_ao x n_mo orbital coefficients (occupied first).  Replaces
 * ccsd_gpu_set_cholesky_mo; the factorisation of S, the triangular solve and both transformation
 * products run on the device. */
int ccsd_gpu_set_cholesky_ao(void *ctx, int64_t n_ao, const double *W_ao, const double *S, const double *C);
/* MO one-electron Hamiltonian h (n_mo x n_mo), orbital energies (n_mo) and E_HF
 * (get_t1_oei, src/wavefunctions/ccs/oei_ccs.F90:35-95; wf%orbital_energies; wf%hf_energy). */
int ccsd_gpu_set_h_mo(void *ctx, const double *h, const double *eps, double e_hf);

/* set_amplitudes + construct_t1_cholesky (src/wavefunctions/ccs/t1_ccs.F90:208-499)
 * + construct_fock (src/wavefunctions/ccsd/fock_ccsd.F90:34-78). */
int ccsd_gpu_set_amplitudes(void *ctx, const double *t);
int ccsd_gpu_get_amplitudes(void *ctx, double *t);
/* set_initial_amplitudes_guess without restart: t1 = 0, t2 = MP2 guess
 * (src/wavefunctions/ccsd/ccsd_class.F90:357-410, 478-533). */
int ccsd_gpu_mp2_guess(void *ctx);
/* T1 Fock matrix F (n_mo x n_mo) at the current amplitudes (wf%fock_ij/ia/ai/ab). */
int ccsd_gpu_get_fock(void *ctx, double *F);

/* calculate_energy (src/wavefunctions/ccsd/mean_value_ccsd.F90:36-99). */
int ccsd_gpu_energy(void *ctx, double *energy);
/* construct_omega (src/wavefunctions/ccsd/omega_ccsd.F90:39-110): omega has n_t1 + n_t2 entries. */
int ccsd_gpu_omega(void *ctx, double *omega);
/* Same with device pointers (output stays in HBM). */
int ccsd_gpu_omega_device(void *ctx, double *d_omega);

/* jacobian_transformation (src/wavefunctions/ccsd/jacobian_ccsd.F90:74-176):
 * rho_k = A c_k for n_vec column vectors (column-major (n_t1+n_t2, n_vec)). */
int ccsd_gpu_jacobian(void *ctx, int64_t n_vec, const double *c, double *rho);
/* jacobian_transpose_transformation (src/wavefunctions/ccsd/jacobian_transpose_ccsd.F90:129-235):
 * sigma_k = b_k^T A. */
int ccsd_gpu_jacobian_transpose(void *ctx, int64_t n_vec, const double *b, double *sigma);

/* The same two transformations on device pointers (trial and result blocks stay in HBM). */
int ccsd_gpu_jacobian_device(void *ctx, int64_t n_vec, const double *d_c, double *d_rho);
int ccsd_gpu_jacobian_transpose_device(void *ctx, int64_t n_vec, const double *d_b, double *d_sigma);

/* prepare_for_jacobian / prepare_for_jacobian_transpose (src/wavefunctions/ccsd/jacobian_ccsd.F90:46-71,
 * jacobian_transpose_ccsd.F90:44-126): side 0 (right) or 1 (left) keeps the intermediates of the
 * current amplitudes that every transformation of a Davidson run reuses (the recorded residual
 * with its primal values, and the transformations' ladder integrals), so later calls of
 * ccsd_gpu_jacobian(_transpose)(_device) only run the derivative pass.  Both sides share what is
 * kept.  Anything that changes the amplitudes, the integrals or the arithmetic (set_amplitudes,
 * set_cholesky_*, set_h_mo, mp2_guess, set_precision, solve_gs) drops it, and the transformations
 * then record afresh per call as without preparation; side -1 drops it explicitly.  Costs the device
 * memory of the recorded residual (about 25 (o v)^2 doubles). */
int ccsd_gpu_prepare_jacobian(void *ctx, int32_t side);

/* Vector-Jacobian product of the residual: given a cotangent b (n_t1 + n_t2), returns
 *   dt = (dOmega/dt)^T b                      (n_t1 + n_t2; sigma = D dt with D = 2 on the doubles diagonal),
 *   dL = (dOmega/dL_mo)^T b  (nullable)       ((J, p, q) over the full MO range, as ccsd_gpu_set_cholesky_mo),
 *   dh = (dOmega/dh_mo)^T b  (nullable)       (n_mo x n_mo).
 * No eT routine returns the L and h parts; they are the density-like contributions of the adjoint. */
int ccsd_gpu_vjp(void *ctx, const double *b, double *dt, double *dL, double *dh);

/* Unrelaxed CCSD one-electron density in the MO basis of h (n_mo x n_mo, column-major):
 *   D_pq = d(E + tbar^T Omega)/dh_pq  at the current amplitudes, orbitals held fixed,
 * i.e. the reference part, the singles part 2 t_ai and tbar^T dOmega/dh (ccsd_gpu_vjp).  With t
 * converged and tbar from ccsd_gpu_solve_multipliers, sum_pq V_pq D_pq is the first-order energy
 * response to h -> h + V (a dipole moment for V = the dipole integrals).  eT builds the same
 * density in the T1 basis (construct_gs_density_doubles, mean_value_doubles.F90:78-114):
 * D_T1 = (1 + t1^T) D (1 - t1^T), with t1 placed in the (virtual, occupied) block. */
int ccsd_gpu_one_electron_density(void *ctx, const double *tbar, double *D);

typedef struct ccsd_gpu_davidson_options {
    int32_t max_iterations;      /* default 100 */
    int32_t block;               /* trial vectors per batched transformation (0 = by memory) */
    int32_t max_reduced_dim;     /* default max(100, 10 n_states), as eT (cc_es_amplitudes_solver_factory_class.F90:307) */
    int32_t start_from_vectors;  /* 1: the `vectors` argument holds start vectors on entry (e.g. a mixed-precision solution) */
    double residual_threshold;   /* |A x - w x| */
    double energy_threshold;     /* |w - w_previous| */
    int32_t reserved[8];
} ccsd_gpu_davidson_options;

/* eigen_davidson_solver%run (src/solvers/eigen_davidson_solver_class.F90:122-229) on the device:
 * the n_states lowest EOM-CCSD excitation energies of A (side 0, right) or A^T (side 1, left) at
 * the current amplitudes.  omega (n_states) on the host; vectors (nullable, host,
 * (n_t1 + n_t2) x n_states) receive the normalised eigenvectors. */
int ccsd_gpu_eom_davidson(void *ctx, int32_t n_states, int32_t side, const ccsd_gpu_davidson_options *opt,
                          double *omega, double *vectors, int32_t *iterations);

/* construct_eta (src/wavefunctions/ccsd/multiplier_equation_ccsd.F90:50-113) at the current amplitudes:
 * eta = [2 F_ia ; packed 4 g_iajb - 2 g_ibja] (n_t1 + n_t2, host). */
int ccsd_gpu_construct_eta(void *ctx, double *eta);

/* Multiplier (Lambda) equations A^T tbar = -eta by linear Davidson on the device (eT's default
 * multiplier solver, src/solvers/linear_davidson_solver_class.F90), started from t1bar = t1,
 * t2bar = packed 2 t_aibj - t_ajbi.  tbar (host, n_t1 + n_t2). */
int ccsd_gpu_solve_multipliers(void *ctx, const ccsd_gpu_davidson_options *opt, double *tbar, int32_t *iterations);

/* run_diis_cc_gs (src/solvers/cc/diis_cc_gs_class.F90:209-315) with the quasi-Newton updater,
 * entirely on the device.  On exit the context holds the final amplitudes; history (nullable)
 * receives max_iterations pairs (E, |Omega|). */
int ccsd_gpu_solve_gs(void *ctx, const ccsd_gpu_solver_options *opt, double *energy,
                      int32_t *iterations, double *history);

/* Counters since creation: kernels of this library launched and GEMM flops issued. */
int ccsd_gpu_stats(void *ctx, int64_t *kernel_launches, double *gemm_flops);

/* Residual evaluations (construct_omega and the solver's) as CUDA graphs: the first evaluation in a
 * precision runs eagerly, later ones replay a graph captured for the same Cholesky vectors, caches
 * and GEMM settings.  Off by default (on when the environment sets CCSD_GPU_GRAPHS=1): capture,
 * instantiation and the graph's own memory cost 5-50 ms per context on a B200, which a solve of
 * 5-16 iterations does not win back except for the smallest systems.  Switching off releases the
 * captured graphs.  No counterpart in eT, which calls BLAS per contraction. */
int ccsd_gpu_set_graphs(void *ctx, int32_t on);

/* FP64 products of at least min_flops flops (<= 0: 1e10; then also 256 in every dimension; 1:
 * every product) on the int8 tensor cores: digits = 4..7 cuts each operand row / column into that many 7-bit int8 digits after a power-of-two
 * scaling (Ozaki's error-free splitting), sums the digit products of weight >= 2^(-7(digits+1))
 * exactly in int32 (tcgen05 kind::i8) and in FP64 in the epilogue; 7 digits reproduce DGEMM to ~1e-14
 * of the largest output.  0 (the default) keeps cuBLAS DGEMM.  Applies to FP64-precision work of the
 * context (the residual, transformations, and the solver's FP64 evaluations unless
 * ccsd_gpu_solver_options.refresh_digits says otherwise).  No counterpart in eT. */
int ccsd_gpu_set_fp64_digits(void *ctx, int32_t digits, double min_flops);

/* Integrals of the FP64 residual.  resident = 1 (the default unless the environment sets
 * CCSD_GPU_FP64_RESIDENT=0): the A2 ladder's +/- pair integrals and the ovvv block of the
 * untransformed Cholesky vectors are formed once per Cholesky set and kept on the device when they
 * fit in half of the free memory (50 GB at o = 32, v = 320), and the T1 transformation enters
 * through o^2 v^3 corrections; resident = 0: the T1-transformed integrals are formed in blocks in
 * every call, as omega_ccsd_a2 does (omega_ccsd.F90:113-480).  Switching off releases them. */
int ccsd_gpu_set_fp64_integrals(void *ctx, int32_t resident);

/* Per-term device times under eT's timing labels ('Construct CCSD Omega', 'omega ccsd a2',
 * 'omega ccsd c2 and d2', 'T1 transform cholesky', 'Jacobian CCSD transformation', ...; eT writes
 * them to eT.timing.out, timings_class.F90:20-80).  on != 0 starts a fresh log (CUDA events around
 * each term on the context's stream; nothing is recorded inside a captured graph), 0 stops it.
 * The report is a JSON object {label: {"calls": n, "ms": total}} written to json (NUL-terminated,
 * truncated to capacity); *needed receives the full length + 1. */
int ccsd_gpu_set_term_timing(void *ctx, int32_t on);
int ccsd_gpu_term_timing_report(void *ctx, char *json, int64_t capacity, int64_t *needed);

/* Residual evaluations served by a graph launch since creation, and the number of GEMM routes the
 * process holds (timed, or loaded from CCSD_GPU_TUNE_FILE). */
int ccsd_gpu_graph_stats(void *ctx, int64_t *residual_replays, int64_t *tuned_routes);

/* Kernel timing: when enabled, every tensor-core GEMM launch is bracketed by CUDA events on the
 * context's stream.  ccsd_gpu_gemm_profile returns the launches recorded since it was enabled,
 * their summed device time (ms) and the tensor flops they issued (3 products x 2mnk). */
int ccsd_gpu_set_profiling(void *ctx, int32_t on);
int ccsd_gpu_gemm_profile(void *ctx, int64_t *launches, double *device_ms, double *tensor_flops);
/* The same for the int8 digit GEMM of FP64-accurate products (ccsd_gpu_set_fp64_digits): launches,
 * summed device time (ms) and int8 tensor ops issued (2mnk per digit product). */
int ccsd_gpu_digit_gemm_profile(void *ctx, int64_t *launches, double *device_ms, double *int8_ops);

/* Diagnostics: C (m x n, column-major, host) = alpha op(A) op(B) + beta C on the device, through
 * the FP64 DGEMM (mixed = 0) or the split-BF16 tcgen05 GEMM that the contractions use (mixed = 1,
 * two bf16 planes), or the three-plane variant of that GEMM (mixed = 2; 6 products, operand rounding
 * 2^-24; not used by the contractions because the FP32 accumulation in the tensor cores, not the
 * operand split, limits their accuracy at CCSD's long K), or the FP64-accurate int8 digit GEMM with
 * mixed = 4..7 digits of 7 bits per operand (tcgen05 kind::i8, exact int32 accumulation). */
int ccsd_gpu_selftest_gemm(void *ctx, int32_t mixed, int32_t transA, int32_t transB, int64_t m, int64_t n,
                           int64_t k, double alpha, const double *A, int64_t lda, const double *B, int64_t ldb,
                           double beta, double *C, int64_t ldc);

/* Allocation-free split-BF16 tensor-core GEMM; no counterpart in eT.
 * C (m x n, column-major, device) = alpha op(A) op(B) + beta C with A, B, C device pointers on the
 * current device, run on `stream` (a cudaStream_t as void*, NULL = legacy default stream).  It is
 * for callers that cannot allocate device memory when they call in (a host program that reserved
 * the whole GPU for its own pool, or a code path that must avoid the synchronisation of
 * cudaMalloc/cudaFree): it makes no cudaMalloc/cudaFree or other allocating call.  Its scratch is a
 * fixed 16 MiB device array inside the library (held by every GPU that loads it):
 * 2 x (round_up(m,128) + round_up(n,256)) x round_up(k,64) must not exceed 8388608, and m, n, k
 * must be below 2^31; larger sizes are rejected with CCSD_GPU_EINVAL.  The call is synchronous: it
 * waits for `stream` to finish the product and reads the GEMM's error word before it returns
 * (CCSD_GPU_ETIMEOUT if a bounded wait ran out), so it must not be called while a stream is being
 * captured into a graph.  The first call on a device looks up the device addresses of the scratch
 * and of the error word.  All calls share the array, so calls that overlap on the GPU (e.g. from two
 * host threads on two streams) race; serialise them.  Errors are reported through
 * ccsd_gpu_last_error(NULL). */
int ccsd_gpu_mixed_gemm_noalloc(int32_t transA, int32_t transB, int64_t m, int64_t n, int64_t k, double alpha,
                                const double *A, int64_t lda, const double *B, int64_t ldb, double beta, double *C,
                                int64_t ldc, void *stream);

/* Diagnostics of the failure path: one m x n x k tensor-core GEMM on the context's stream in which
 * the TMA producer withholds the loads of its first pipeline stage, so the MMA warp's bounded wait
 * for them runs out by design after wait_cycles SM clock cycles (<= 0: the normal bound, ~2 s).
 * Returns CCSD_GPU_ETIMEOUT when the kernel reported the time-out as designed; the context stays
 * usable afterwards.  No counterpart in eT. */
int ccsd_gpu_selftest_gemm_stall(void *ctx, int64_t m, int64_t n, int64_t k, int64_t wait_cycles);

/* Algorithmic flop count of one Omega at this context's dimensions, summed over eT's own BLAS
 * call sites (2mnk per DGEMM, n(n+1)k per DSFRK). */
double ccsd_gpu_omega_flops(void *ctx);

/* One independent system of a batch: host arrays in the layouts of ccsd_gpu_set_cholesky_mo and
 * ccsd_gpu_set_h_mo. */
typedef struct ccsd_gpu_batch_system {
    int64_t n_o, n_v, n_J;
    const double *L_mo;          /* (J, n_mo, n_mo) column-major */
    const double *h_mo;          /* n_mo x n_mo */
    const double *eps;           /* n_mo orbital energies */
    double e_hf;
    double *t_out;               /* optional: the final amplitudes (n_t1 + n_t2), or NULL */
} ccsd_gpu_batch_system;

/* Ground states of many independent systems of uneven size.  eT runs one wavefunction per process
 * and has no such entry point; this is the batch of the uneven-batch workload.  `workers` host
 * threads (1..64) each take the next system (largest o^2 v^4 first), create a context on
 * opt->device with its own stream, start from the MP2 guess, run ccsd_gpu_solve_gs with `sopt` and
 * release the context, so the kernels of systems in flight overlap on the GPU.  Per system the
 * energy, iteration count and status are written (arrays of n_systems, each may be NULL); the
 * return value is CCSD_GPU_OK when every system converged, else the first non-zero status in
 * system order.  Device memory in use is that of `workers` systems at a time. */
int ccsd_gpu_solve_gs_batch(int32_t n_systems, const ccsd_gpu_batch_system *systems, const ccsd_gpu_options *opt,
                            const ccsd_gpu_solver_options *sopt, int32_t workers, double *energies,
                            int32_t *iterations, int32_t *status);

#ifdef __cplusplus
}
#endif

#endif /* CCSD_GPU_H */
