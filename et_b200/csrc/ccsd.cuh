// The per-system context behind the C ABI.
#pragma once

#include <memory>
#include <string>

#include "common.cuh"
#include "ozaki_gemm.cuh"
#include "graph.cuh"

namespace ccsd {

// node ids of the recorded residual
struct OmegaNodes {
    int t1, t2, L_oo, L_ov, L_vo, L_vv, h_oo, h_ov, h_vo, h_vv, Lt_vv, om1, om2;
};

// The residual recorded once at the current amplitudes for all Jacobian transformations of a
// Davidson run (prepare_for_jacobian, jacobian_ccsd.F90:46-71): its primal values, and through its
// ladder op the Y intermediate and the transposed vectors; valid for the arithmetic it was
// recorded with and until the amplitudes, integrals or h change.
struct PreparedJacobian {
    std::unique_ptr<Graph> g;
    OmegaNodes n{};
    Prec prec = Prec::FP64;
    int planes = 0;
    int64_t k_chunk = 0, l_version = -1;
    int64_t id = -1;
};

struct Context {
    int64_t no, nv, nJ, nmo, nov, nt1, nt2, namp;
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cublasHandle_t blas = nullptr;
    Exec ex;
    GemmProfile prof;
    TermLog terms;                  // per-term device times under eT's labels (ccsd_gpu_set_term_timing)
    int64_t ladder_batch = 0;
    int64_t ladder_pair_budget = 0;  // bytes the resident split-bf16 pair integrals may take (0 = automatic)
    double e_hf = 0.0;
    bool have_L = false, have_h = false, have_t = false;
    std::string err;

    // Device buffers are stream-ordered allocations on the context's stream: ~Context() releases
    // each of them before it destroys that stream, so a new resident buffer joins its list.
    // MO Cholesky blocks (J, p, q) and their T1-transformed counterparts
    DBuf L_oo, L_ov, L_vo, L_vv;
    DBuf Lt_oo, Lt_ov, Lt_vo, Lt_vv;
    DBuf h, eps, F;          // h_mo, orbital energies, T1 Fock (n_mo x n_mo)
    DBuf fb_oo, fb_ov, fb_vo, fb_vv;   // the T1 Fock matrix in o/v blocks (contiguous)
    // Lt_* and F hold the T1 transformation of the current t1 (set by refresh(), cleared when the
    // solver moves t): the plain residual then takes them as inputs instead of recording them
    bool t1_current = false;
    DBuf hb_oo, hb_ov, hb_vo, hb_vv;   // MO h in o/v blocks
    DBuf t;                  // [t1 | packed t2]
    DBuf epsdiff;            // orbital differences (n_amp)
    DBuf scal;               // scalar scratch
    DBuf mbuf;               // split-bf16 ladder integrals g+- of all pairs, P+ then P- (mixed precision)
    size_t mbuf_bytes = 0;
    DBuf gov;                  // g_iajb cache (g_ovov_const)
    bool have_gov = false;
    int64_t gov_id = 0;        // bumped whenever gov is formed again
    DBuf hov;                  // g_lckd - 1/2 g_kcld (h_ovov_const), formed from gov number hov_id
    int64_t hov_id = -1;
    int64_t l_version = 0;     // bumped whenever the Cholesky vectors change
    // what mbuf holds: 0 nothing, 1 untransformed L_vv pairs (valid for mbuf_version), 2 per call
    int mbuf_kind = 0, mbuf_planes = 0;
    int64_t mbuf_version = -1;
    // split-bf16 ovvv integrals g_kcbd of the untransformed vectors at [plane][k + no*b][c + nv*d]
    // (mixed precision; valid for ybuf_version)
    DBuf ybuf;
    size_t ybuf_bytes = 0;
    int ybuf_planes = 0;
    int64_t ybuf_version = -1;
    int ybuf_fit = -1;              // residency decision for (ybuf_fit_version, ybuf_fit_planes)
    int64_t ybuf_fit_version = -1;
    int ybuf_fit_planes = 0;
    // FP64 residual with resident integrals of the untransformed vectors (when they fit): eT's +/-
    // ladder integrals g+ [v(v+1)/2 x v(v+1)/2] and g- [v(v-1)/2 x v(v-1)/2] for all pairs, and the
    // ovvv block g_kcbd as [k, b, c, d]; valid for f64_version
    DBuf f64_gp, f64_gm, f64_ovvv;
    int64_t f64_version = -1;
    int f64_fit = -1;               // residency decision for f64_fit_version
    int64_t f64_fit_version = -1;
    bool f64_resident_on = true;    // CCSD_GPU_FP64_RESIDENT=0 keeps eT's per-call integrals
    // bumped whenever a resident cache (g_iajb, ladder pair integrals, ovvv planes) is (re)built, so
    // a captured residual that points into the old one is not replayed
    int64_t cache_epoch = 0;
    DBuf blas_ws;                   // cuBLAS workspace (no allocation inside stream capture)
    DBuf gemm_err;                  // error word of this context's tensor-core GEMMs (ex.gemm_err)
    DBuf digit_arena;               // scratch of the int8 digit GEMM (ex.digit_arena), grow-only
    // ccsd_gpu_prepare_jacobian: the recorded residual shared by the transformations, and the id
    // under which the ladder integrals a prepared transformation forms stay in mbuf for the next one
    std::unique_ptr<PreparedJacobian> prep;
    int64_t prep_counter = 0;
    int64_t pairs_reuse_id = -1;    // the prepared id while a prepared transformation runs, else -1
    const double *mbuf_src = nullptr;   // the L_vv whose pair integrals mbuf holds (mbuf_kind 2)
    int64_t mbuf_reuse = -1;            // the prepared id they were formed for

    // The residual evaluation captured as a CUDA graph, one per precision.  The first evaluation in
    // a precision runs eagerly (it builds the caches and times the GEMM routes); later ones replay
    // a graph captured for the same Cholesky set, caches and GEMM settings, which writes om_stage.
    struct ResidualGraph {
        cudaGraphExec_t exec = nullptr;
        bool warm = false;
        int64_t l_version = -1, cache_epoch = -1, k_chunk = 0;
        int planes = 0;
        int64_t launches = 0;
        double flops = 0.0;
        void reset() {
            if (exec) cudaGraphExecDestroy(exec);
            exec = nullptr;
        }
    };
    ResidualGraph rgraph[2];        // [0] FP64, [1] MIXED
    DBuf om_stage;                  // the residual graphs' output
    bool use_graphs = false;        // ccsd_gpu_set_graphs or CCSD_GPU_GRAPHS=1 turns capture on
    int64_t graph_replays = 0;      // residual evaluations served by a graph launch
    bool graphs_captured = false;

    Context(int64_t no, int64_t nv, int64_t nJ, const ccsd_gpu_options *opt);
    ~Context();

    void set_stream(cudaStream_t s);
    void t1_transform_cholesky();
    void construct_fock();
    void refresh();                        // T1 transformation + Fock at the current t
    void set_precision(int32_t precision);   // CCSD_GPU_FP64 / CCSD_GPU_MIXED
    DBuf g_ovov();
    // g_iajb = sum_J L_ia L_jb in FP64, kept until the Cholesky vectors change: the ov block is
    // unchanged by the T1 transformation, so every iteration shares it
    const double *g_ovov_const();
    const double *h_ovov_const();
    double energy();
    void mp2_guess();
    void omega(double *d_omega);
    void omega_eager(double *d_omega);       // record + evaluate the residual on ex.stream
    void prepare_residual_caches();          // builds what a captured residual only reads
    void capture_residual(ResidualGraph &G, double *d_omega);
    // const_ovov: take g_iajb from the cache (no derivative flows into L_ov through it)
    // const_t1: take the T1-transformed blocks and the Fock matrix from the context (only when no
    // derivative will be taken and t1_current holds)
    OmegaNodes record_omega(Graph &g, bool const_ovov = true, bool const_t1 = false);
    void record_ladder(Graph &g, int om2, int Lvv, int t2, int t1, int L_vv_in, int tf);
    void ladder_y(const double *Lvv, const double *tfull, double *Y);
    // mixed precision: whether the resident ovvv planes fit, their construction, and
    // Y0_kibj = sum_cd g_kcbd tau_cidj from them
    bool ovvv_resident();
    void ovvv_pairs();
    void ladder_y0(const double *tfull, double *Y);
    // Y with the T1-transformed vv block Ltvv, sum_cd g_kc~bd tau_cidj: in mixed precision
    // Y0_kibj - sum_l t_bl Q_kilj (Q_kilj = sum_cd g_kcld tau_cidj), else ladder_y(Ltvv)
    void ladder_y_t1(const double *t1, const double *Ltvv, const double *tfull, double *Y);
    // throws CCSD_GPU_ETIMEOUT (and clears the word) when a tensor-core GEMM of this context
    // reported a bounded wait that ran out
    void check_gemm();
    void prepare_jacobian();
    void drop_jacobian();
    // the prepared recording when it is valid for the current arithmetic, else a fresh recording
    // into `local`
    Graph &transform_graph(std::unique_ptr<Graph> &local, OmegaNodes &n);
    void jacobian(int64_t nvec, const double *c, double *rho);
    void jacobian_transpose(int64_t nvec, const double *b, double *sigma);
    void adjoint(const double *b, double *dt, double *dL, double *dh);
    void set_h_blocks();
    // A2 ladder: om2[v] += ladder(L_vv in (J, a, c) layout, packed t2[v]) for nvec vectors (stride
    // n_t2); the integrals are formed once per call
    void ladder(const double *Lvv, const double *t2, double *om2, int64_t nvec = 1);
    void ladder_tc(const double *Lvv, const double *t2, double *om2, int64_t nvec, bool untransformed);
    DBuf lvv_jca(const double *Lvv);
    void form_pair_planes(const double *LT, int64_t a0, int64_t a1, double *G, __nv_bfloat16 *Pp, int64_t rows_p,
                          int64_t rowp0, __nv_bfloat16 *Pm, int64_t rows_m, int64_t rowm0);
    bool ladder_pairs_resident();
    void ladder_tc_streamed(const double *Lvv, const double *t2, double *om2, int64_t nvec);
    void ladder_pairs(const double *Lvv, bool untransformed);
    struct TPlanes {
        DBuf p, m;                   // t+ and t- planes
        int64_t rows_p = 0, rows_m = 0;
    };
    TPlanes t_planes(const double *t2, int64_t nvec);
    void ladder_pm_block(const TPlanes &T, int64_t nvec, const __nv_bfloat16 *Pp, int64_t prow, const __nv_bfloat16 *Pm,
                         int64_t mrow, int64_t a0, int64_t a1, double *om2);
    // the residual's ladder in mixed precision from untransformed integrals plus t1 corrections
    void ladder_residual_mixed(const double *t1, const double *tf, const double *t2, double *om2);
    // om2 += pack(-(A + A^T) + T4) with A_aibj = sum_k t_ak Y0_kibj, T4 = sum_kl t_ak t_bl Q_kilj
    void ladder_t1_corrections(const double *t1, const double *tf, const double *Y0, double *om2);
    // the same ladder in FP64 from resident FP64 integrals (f64_resident() must hold)
    bool f64_resident();
    void f64_integrals();
    void ladder_residual_f64(const double *t1, const double *tf, const double *t2, double *om2);
    // digit planes of the resident FP64 integrals for FP64 evaluations on the int8 digit GEMM: the
    // +/- ladder integrals (B operands) and g_kcbd (A operand of Y), kept per Cholesky set and digit
    // count while they fit (levels: 2 all three, 1 the ladder pair only, 0 none)
    int f64_digit_planes(int digits);
    OzPlanes f64_gp_dig, f64_gm_dig, f64_ovvv_dig;
    int64_t f64_dig_version = -1;
    int f64_dig_digits = 0, f64_dig_level = 0;
    int davidson(int nstates, int side, const ccsd_gpu_davidson_options *o, double *omega_out, double *vectors_out,
                 int32_t *iters_out, const double *start = nullptr);
    void eta(double *out);
    int multipliers(const ccsd_gpu_davidson_options *o, double *tbar, int32_t *iters_out);
    int solve_gs(const ccsd_gpu_solver_options *o, double *energy, int32_t *iters, double *history);
    double omega_flops() const;
};

}  // namespace ccsd
