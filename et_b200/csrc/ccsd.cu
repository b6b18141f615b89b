// CCSD hot path on one B200: T1-transformed Cholesky vectors, T1 Fock matrix, energy,
// the residual Omega(t), and the device-resident quasi-Newton + DIIS ground-state solver.
// Each step restates one eT routine (paths relative to the eT source tree).
#include <cuda_bf16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>

#include "autotune.cuh"
#include "ccsd.cuh"
#include "ccsd_kernels.cuh"
#include "mixed_gemm.cuh"
#include "tensor_ops.cuh"

namespace ccsd {

Context::Context(int64_t no_, int64_t nv_, int64_t nJ_, const ccsd_gpu_options *opt)
    : no(no_), nv(nv_), nJ(nJ_) {
    REQUIRE(no > 0 && nv > 0 && nJ > 0, CCSD_GPU_EINVAL, "dimensions must be positive");
    nmo = no + nv;
    nov = no * nv;
    nt1 = nov;
    nt2 = nov * (nov + 1) / 2;
    namp = nt1 + nt2;
    device = opt ? opt->device : 0;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        throw Error(CCSD_GPU_ENODEV, "no CUDA device available");
    REQUIRE(device >= 0 && device < ndev, CCSD_GPU_EINVAL, "device ordinal out of range");
    CU_CHECK(cudaSetDevice(device));
    cudaDeviceProp prop;
    CU_CHECK(cudaGetDeviceProperties(&prop, device));
    REQUIRE(prop.major == 10, CCSD_GPU_ENODEV,
            std::string("this library is built for sm_100a; device is sm_") + std::to_string(prop.major) +
                std::to_string(prop.minor));
    cudaMemPool_t pool;
    CU_CHECK(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t thr = UINT64_MAX;
    CU_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    CU_CHECK(cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking));
    BLAS_CHECK(cublasCreate(&blas));
    set_stream(nullptr);
    {
        // cuBLAS works in a buffer it is given, so its calls can be captured into a graph
        const size_t ws = size_t(32) << 20;
        blas_ws = DBuf(ws, own_stream);
        CU_CHECK(cudaStreamSynchronize(own_stream));
        BLAS_CHECK(cublasSetWorkspace(blas, blas_ws.as<void>(), ws));
        const char *g = std::getenv("CCSD_GPU_GRAPHS");
        use_graphs = g && g[0] == '1';
        const char *r = std::getenv("CCSD_GPU_FP64_RESIDENT");
        f64_resident_on = !(r && r[0] == '0');
        // digits of the first-order FP64 terms of the mixed residual: CCSD_GPU_MIXED_FP64_DIGITS=0 keeps
        // them on cuBLAS DGEMM
        if (const char *d = std::getenv("CCSD_GPU_MIXED_FP64_DIGITS")) {
            const int v = std::atoi(d);
            ex.mixed_fp64_digits = (v >= 4 && v <= 7) ? v : 0;
        }
    }
    ex.blas = blas;
    ex.prof = &prof;
    ex.terms = &terms;
    gemm_err = DBuf(sizeof(int), own_stream);
    CU_CHECK(cudaMemsetAsync(gemm_err.as<void>(), 0, sizeof(int), own_stream));
    ex.gemm_err = gemm_err.as<int>();
    ex.digit_arena = &digit_arena;
    set_precision(opt ? opt->precision : CCSD_GPU_FP64);
    if (opt && opt->mixed_min_flops > 0) ex.mixed_min_flops = (double)opt->mixed_min_flops;
    if (opt && opt->mixed_k_chunk != 0) ex.k_chunk = opt->mixed_k_chunk;
    {
        const char *env = std::getenv("CCSD_GPU_AUTOTUNE");
        const int64_t at = opt ? opt->autotune : 0;
        ex.autotune = at > 0 || (at == 0 && !(opt && opt->mixed_min_flops > 0) && !(env && env[0] == '0'));
    }
    ladder_batch = opt ? opt->ladder_batch : 0;
    ladder_pair_budget = opt ? opt->ladder_pair_budget : 0;
    cudaStream_t s = ex.stream;
    for (auto *b : {&L_oo, &Lt_oo}) *b = dalloc(nJ * no * no, s);
    for (auto *b : {&L_ov, &Lt_ov}) *b = dalloc(nJ * no * nv, s);
    for (auto *b : {&L_vo, &Lt_vo}) *b = dalloc(nJ * nv * no, s);
    for (auto *b : {&L_vv, &Lt_vv}) *b = dalloc(nJ * nv * nv, s);
    h = dalloc(nmo * nmo, s);
    hb_oo = dalloc(no * no, s);
    hb_ov = dalloc(no * nv, s);
    hb_vo = dalloc(nv * no, s);
    hb_vv = dalloc(nv * nv, s);
    eps = dalloc(nmo, s);
    F = dalloc(nmo * nmo, s);
    fb_oo = dalloc(no * no, s);
    fb_ov = dalloc(no * nv, s);
    fb_vo = dalloc(nv * no, s);
    fb_vv = dalloc(nv * nv, s);
    t = dalloc(namp, s);
    epsdiff = dalloc(namp, s);
    scal = dalloc(64, s);
    fill(ex, t.d(), namp, 0.0);
    CU_CHECK(cudaStreamSynchronize(s));
}

Context::~Context() {
    if (own_stream) cudaStreamSynchronize(own_stream);
    if (ex.stream && ex.stream != own_stream) cudaStreamSynchronize(ex.stream);
    // every device buffer is freed (stream-ordered) while its stream still exists
    prep.reset();
    for (auto &G : rgraph) G.reset();
    if (ex.stream) cudaStreamSynchronize(ex.stream);
    if (graphs_captured) cudaDeviceGraphMemTrim(device);   // the physical memory the residual graphs held
    for (OzPlanes *p : {&f64_gp_dig, &f64_gm_dig, &f64_ovvv_dig}) p->buf.release();
    for (DBuf *b : {&gov, &hov, &L_oo, &L_ov, &L_vo, &L_vv, &Lt_oo, &Lt_ov, &Lt_vo, &Lt_vv, &h, &eps, &F, &t, &epsdiff, &scal,
                    &mbuf, &ybuf, &om_stage, &f64_gp, &f64_gm, &f64_ovvv, &hb_oo, &hb_ov, &hb_vo, &hb_vv,
                    &gemm_err, &digit_arena, &fb_oo, &fb_ov, &fb_vo, &fb_vv})
        b->release();
    if (blas) cublasDestroy(blas);
    blas = nullptr;
    blas_ws.release();
    mbuf_bytes = 0;
    ybuf_bytes = 0;
    if (ex.stream) cudaStreamSynchronize(ex.stream);
    prof.clear();
    terms.clear();
    if (blas) cublasDestroy(blas);
    if (own_stream) {
        cudaStreamSynchronize(own_stream);
        cudaStreamDestroy(own_stream);
    }
}

void Context::set_stream(cudaStream_t s) {
    ex.stream = s ? s : own_stream;
    BLAS_CHECK(cublasSetStream(blas, ex.stream));
}

// ---------------------------------------------------------------------------
// T1 transformation of the Cholesky vectors (src/wavefunctions/ccs/t1_ccs.F90:208-499)
// ---------------------------------------------------------------------------
void Context::t1_transform_cholesky() {
    const double *t1 = t.d();
    TV T1 = tv(t1, {nv, no});
    cudaStream_t s = ex.stream;
    // ov block unchanged
    CU_CHECK(cudaMemcpyAsync(Lt_ov.d(), L_ov.d(), sizeof(double) * nJ * no * nv, cudaMemcpyDeviceToDevice, s));
    // oo: L_ij + sum_a L_ia t_aj                                   (:251-290)
    CU_CHECK(cudaMemcpyAsync(Lt_oo.d(), L_oo.d(), sizeof(double) * nJ * no * no, cudaMemcpyDeviceToDevice, s));
    contract(ex, "Jia,aj->Jij", 1.0, tv(L_ov.d(), {nJ, no, nv}), T1, 1.0, tv(Lt_oo.d(), {nJ, no, no}));
    // vo: L_ai + sum_b L_ab t_bi - sum_j t_aj (L_ji + sum_b L_jb t_bi) (:293-440); the bracket is Lt_oo
    CU_CHECK(cudaMemcpyAsync(Lt_vo.d(), L_vo.d(), sizeof(double) * nJ * nv * no, cudaMemcpyDeviceToDevice, s));
    contract(ex, "Jab,bi->Jai", 1.0, tv(L_vv.d(), {nJ, nv, nv}), T1, 1.0, tv(Lt_vo.d(), {nJ, nv, no}));
    // - sum_j Lt_oo[J, j, i] t_aj for each i: [J x j] times t1^T, written in place ((J, a) of one i is
    // one contiguous block of Lt_vo, so no reordered copy of the output is needed)
    gemm_batched_f64(ex, false, true, nJ, nv, no, -1.0, Lt_oo.d(), nJ, nJ * no, t1, nv, 0, 1.0, Lt_vo.d(), nJ,
                     nJ * nv, no);
    // vv: L_ab - sum_j t_aj L_jb                                  (:443-499), per b in place likewise
    CU_CHECK(cudaMemcpyAsync(Lt_vv.d(), L_vv.d(), sizeof(double) * nJ * nv * nv, cudaMemcpyDeviceToDevice, s));
    gemm_batched_f64(ex, false, true, nJ, nv, no, -1.0, L_ov.d(), nJ, nJ * no, t1, nv, 0, 1.0, Lt_vv.d(), nJ,
                     nJ * nv, nv);
}

// ---------------------------------------------------------------------------
// T1 Fock matrix F_pq = h~_pq + sum_k (2 g~_pqkk - g~_pkkq)
// (src/wavefunctions/ccsd/fock_ccsd.F90:34-78, src/wavefunctions/ccs/fock_ccs.F90:242-1107)
// ---------------------------------------------------------------------------
void Context::construct_fock() {
    cudaStream_t s = ex.stream;
    double *Fm = F.d();
    TV T1 = tv(t.d(), {nv, no});
    // h~ = X h Y^T, X = 1 - t1, Y = 1 + t1^T (t1_ccs.F90:34-95)
    CU_CHECK(cudaMemcpyAsync(Fm, h.d(), sizeof(double) * nmo * nmo, cudaMemcpyDeviceToDevice, s));
    auto blk = [&](double *base, int64_t r0, int64_t c0, int64_t nr, int64_t nc) {
        TV v;
        v.p = base + r0 + nmo * c0;
        v.nd = 2;
        v.n[0] = nr;
        v.n[1] = nc;
        v.s[0] = 1;
        v.s[1] = nmo;
        return v;
    };
    // rows v: W_aq -= sum_i t_ai h_iq
    contract(ex, "ai,iq->aq", -1.0, T1, blk(h.d(), 0, 0, no, nmo), 1.0, blk(Fm, no, 0, nv, nmo));
    // cols o: W_pi += sum_a W_pa t_ai
    contract(ex, "pa,ai->pi", 1.0, blk(Fm, 0, no, nmo, nv), T1, 1.0, blk(Fm, 0, 0, nmo, no));
    // Coulomb: 2 sum_J L~_pq X_J with X_J = sum_k L~_kk
    DBuf X = dalloc(nJ, s);
    trace_oo(ex, Lt_oo.d(), nJ, no, X.d());
    TV XJ = tv(X.d(), {nJ});
    contract(ex, "Jpq,J->pq", 2.0, tv(Lt_oo.d(), {nJ, no, no}), XJ, 1.0, blk(Fm, 0, 0, no, no));
    contract(ex, "Jpq,J->pq", 2.0, tv(Lt_ov.d(), {nJ, no, nv}), XJ, 1.0, blk(Fm, 0, no, no, nv));
    contract(ex, "Jpq,J->pq", 2.0, tv(Lt_vo.d(), {nJ, nv, no}), XJ, 1.0, blk(Fm, no, 0, nv, no));
    contract(ex, "Jpq,J->pq", 2.0, tv(Lt_vv.d(), {nJ, nv, nv}), XJ, 1.0, blk(Fm, no, no, nv, nv));
    // exchange: - sum_{J,k} L~_pk L~_kq
    contract(ex, "Jpk,Jkq->pq", -1.0, tv(Lt_oo.d(), {nJ, no, no}), tv(Lt_oo.d(), {nJ, no, no}), 1.0,
             blk(Fm, 0, 0, no, no));
    contract(ex, "Jpk,Jkq->pq", -1.0, tv(Lt_oo.d(), {nJ, no, no}), tv(Lt_ov.d(), {nJ, no, nv}), 1.0,
             blk(Fm, 0, no, no, nv));
    contract(ex, "Jpk,Jkq->pq", -1.0, tv(Lt_vo.d(), {nJ, nv, no}), tv(Lt_oo.d(), {nJ, no, no}), 1.0,
             blk(Fm, no, 0, nv, no));
    contract(ex, "Jpk,Jkq->pq", -1.0, tv(Lt_vo.d(), {nJ, nv, no}), tv(Lt_ov.d(), {nJ, no, nv}), 1.0,
             blk(Fm, no, no, nv, nv));
}

void Context::set_h_blocks() {
    auto blk = [&](int64_t r0, int64_t c0, int64_t nr, int64_t nc, double *dst) {
        TV v;
        v.p = h.d() + r0 + nmo * c0;
        v.nd = 2;
        v.n[0] = nr;
        v.n[1] = nc;
        v.s[0] = 1;
        v.s[1] = nmo;
        permute_add(ex, 1.0, v, 0.0, tv(dst, {nr, nc}));
    };
    blk(0, 0, no, no, hb_oo.d());
    blk(0, no, no, nv, hb_ov.d());
    blk(no, 0, nv, no, hb_vo.d());
    blk(no, no, nv, nv, hb_vv.d());
}

void Context::refresh() {
    REQUIRE(have_L && have_h, CCSD_GPU_ESTATE, "Cholesky vectors and h must be set first");
    drop_jacobian();   // the amplitudes (or integrals) the prepared transformations were recorded at are gone
    Prec keep = ex.prec;
    ex.prec = Prec::FP64;      // the T1 transformation and the Fock matrix stay FP64
    {
        TermTimer tt(ex, "T1 transform cholesky");
        t1_transform_cholesky();
    }
    {
        TermTimer tt(ex, "Fock matrix construction (T1 basis)");
        construct_fock();
        auto blk = [&](DBuf &dst, int64_t r0, int64_t c0, int64_t nr, int64_t nc) {
            CU_CHECK(cudaMemcpy2DAsync(dst.d(), sizeof(double) * nr, F.d() + r0 + nmo * c0, sizeof(double) * nmo,
                                       sizeof(double) * nr, nc, cudaMemcpyDeviceToDevice, ex.stream));
        };
        blk(fb_oo, 0, 0, no, no);
        blk(fb_ov, 0, no, no, nv);
        blk(fb_vo, no, 0, nv, no);
        blk(fb_vv, no, no, nv, nv);
    }
    ex.prec = keep;
    t1_current = true;
}

// g_ovov[i,a,j,b] = sum_J L_ia L_jb  (eri_t1%get('ovov'))
DBuf Context::g_ovov() {
    DBuf g = dalloc(nov * nov, ex.stream);
    contract(ex, "Jia,Jjb->iajb", 1.0, tv(Lt_ov.d(), {nJ, no, nv}), tv(Lt_ov.d(), {nJ, no, nv}), 0.0,
             tv(g.d(), {no, nv, no, nv}));
    return g;
}

const double *Context::g_ovov_const() {
    if (!have_gov) {
        const Prec keep = ex.prec;
        ex.prec = Prec::FP64;
        gov = g_ovov();
        ex.prec = keep;
        have_gov = true;
        gov_id++;
        cache_epoch++;
    }
    return gov.d();
}

// H_lckd = g_lckd - 1/2 g_kcld, the combination of g_ovov that the two u terms of omega_ccsd_d2
// contract with (one product instead of two), kept beside g_ovov
const double *Context::h_ovov_const() {
    const double *g = g_ovov_const();
    if (!hov || hov_id != gov_id) {
        if (!hov) hov = dalloc(nov * nov, ex.stream);
        const TV H = tv(hov.d(), {no, nv, no, nv});
        permute_add(ex, 1.0, tv(g, {no, nv, no, nv}), 0.0, H);
        TV gt = tv(g, {no, nv, no, nv});   // gt[l, c, k, d] = g[k, c, l, d]
        std::swap(gt.s[0], gt.s[2]);
        permute_add(ex, -0.5, gt, 1.0, H);
        hov_id = gov_id;
        cache_epoch++;
    }
    return hov.d();
}

// calculate_energy_ccsd (src/wavefunctions/ccsd/mean_value_ccsd.F90:36-99), FP64
double Context::energy() {
    Prec keep = ex.prec;
    ex.prec = Prec::FP64;
    const double *gov_p = g_ovov_const();
    {
        TermTimer tt(ex, "Calculate energy");
        energy_reduce(ex, t.d(), t.d() + nt1, gov_p, no, nv, e_hf, scal.d());
    }
    ex.prec = keep;
    double e;
    CU_CHECK(cudaMemcpyAsync(&e, scal.d(), sizeof(double), cudaMemcpyDeviceToHost, ex.stream));
    CU_CHECK(cudaStreamSynchronize(ex.stream));
    return e;
}

// set_t2_to_cc2_guess (src/wavefunctions/ccsd/ccsd_class.F90:478-533) at t1 = 0
void Context::mp2_guess() {
    fill(ex, t.d(), namp, 0.0);
    refresh();
    orbital_differences(ex, eps.d(), no, nv, epsdiff.d());
    DBuf g = dalloc(nov * nov, ex.stream);
    Prec keep = ex.prec;
    ex.prec = Prec::FP64;
    contract(ex, "Jai,Jbj->aibj", 1.0, tv(Lt_vo.d(), {nJ, nv, no}), tv(Lt_vo.d(), {nJ, nv, no}), 0.0,
             tv(g.d(), {nv, no, nv, no}));
    ex.prec = keep;
    mp2_amplitudes(ex, g.d(), epsdiff.d(), nov, t.d() + nt1);
    have_t = true;
}

// ---------------------------------------------------------------------------
// A2 ladder: Omega^ab_ij += sum_cd g_acbd t^cd_ij with the +/- symmetrisation of
// omega_ccsd_a2 (src/wavefunctions/ccsd/omega_ccsd.F90:113-480), batched over a.
// ---------------------------------------------------------------------------
void Context::ladder(const double *Lvv, const double *t2, double *om2, int64_t nvec) {
    if (nvec <= 0) return;
    if (ex.prec == Prec::MIXED) {
        ladder_tc(Lvv, t2, om2, nvec, false);
        return;
    }
    cudaStream_t s = ex.stream;
    const int64_t nop = no * (no + 1) / 2, nom = no * (no - 1) / 2;
    const int64_t nvp = nv * (nv + 1) / 2, nvm = nv * (nv - 1) / 2;
    // the nvec vectors side by side: rows [v n_o_p, (v+1) n_o_p) of t+ belong to vector v
    const int64_t ldp = nvec * nop, ldm = std::max<int64_t>(nvec * nom, 1);
    DBuf tp = dalloc(ldp * nvp, s), tm = dalloc(ldm * std::max<int64_t>(nvm, 1), s);
    for (int64_t v = 0; v < nvec; v++) build_tpm(ex, t2 + v * nt2, tp.d() + v * nop, tm.d() + v * nom, no, nv, ldp, ldm);
    // L~_vv as (J, c, a): columns (c, a) of one a-block are contiguous
    DBuf LT = dalloc(nJ * nv * nv, s);
    {
        TV src = tv(Lvv, {nJ, nv, nv});   // [J, a, c]
        TV dst;
        dst.p = LT.d();
        dst.nd = 3;
        dst.n[0] = nJ;
        dst.n[1] = nv;
        dst.n[2] = nv;
        dst.s[0] = 1;
        dst.s[1] = nJ * nv;   // a
        dst.s[2] = nJ;        // c
        permute_add(ex, 1.0, src, 0.0, dst);
    }
    // batch length over a: keep G + g+- + w+- within the budget
    int64_t nA = ladder_batch;
    if (nA <= 0) {
        const double budget = 6.0e9;   // bytes
        double per_a = 8.0 * (double)nv * nv * nv + 16.0 * (double)nvp * nv + 16.0 * (double)ldp * nv;
        nA = std::max<int64_t>(1, std::min<int64_t>(nv, (int64_t)(budget / per_a)));
    }
    int64_t maxab = 0;
    for (int64_t a0 = 0; a0 < nv; a0 += nA) {
        int64_t a1 = std::min(nv, a0 + nA);
        maxab = std::max(maxab, a1 * (a1 + 1) / 2 - a0 * (a0 + 1) / 2);
    }
    DBuf G = dalloc(nv * nA * nv * nv, s);
    DBuf gp = dalloc(nvp * maxab, s), gm = dalloc(std::max<int64_t>(nvm * maxab, 1), s);
    DBuf wp = dalloc(ldp * maxab, s), wm = dalloc(ldm * maxab, s);
    for (int64_t a0 = 0; a0 < nv; a0 += nA) {
        int64_t a1 = std::min(nv, a0 + nA);
        int64_t M = nv * (a1 - a0), N = nv * a1;
        // G[(c,a),(d,b)] = sum_J L_ac L_bd   (eri_t1%get('vvvv') / get_packed('vv')), once for all vectors
        gemm(ex, true, false, M, N, nJ, 1.0, LT.d() + nJ * nv * a0, nJ, LT.d(), nJ, 0.0, G.d(), M);
        form_gpm(ex, G.d(), M, gp.d(), gm.d(), nv, a0, a1);
        int64_t nabp = a1 * (a1 + 1) / 2 - a0 * (a0 + 1) / 2;
        int64_t nabm = a1 * (a1 - 1) / 2 - a0 * (a0 - 1) / 2;
        gemm(ex, false, false, ldp, nabp, nvp, 0.5, tp.d(), ldp, gp.d(), nvp, 0.0, wp.d(), ldp);
        if (nom > 0 && nabm > 0)
            gemm(ex, false, false, nvec * nom, nabm, nvm, 0.5, tm.d(), ldm, gm.d(), nvm, 0.0, wm.d(), ldm);
        for (int64_t v = 0; v < nvec; v++)
            add_omega_pm(ex, om2 + v * nt2, wp.d() + v * nop, wm.d() + v * nom, no, nv, a0, a1, ldp, ldm);
    }
}

void Context::set_precision(int32_t precision) {
    REQUIRE(precision == CCSD_GPU_FP64 || precision == CCSD_GPU_MIXED, CCSD_GPU_EINVAL, "unknown precision");
    const Prec p = precision == CCSD_GPU_FP64 ? Prec::FP64 : Prec::MIXED;
    if (p != ex.prec) drop_jacobian();
    ex.prec = p;
}

// Tensor-core form of the same +/- ladder: the FP64 path's g+- (over packed c >= d, c > d) and t+-
// meet in two GEMMs on split-bf16 planes, W+ = 1/2 t+ g+^T (K = n_v(n_v+1)/2) and W- = 1/2 t- g-^T
// (K = n_v(n_v-1)/2): half the work of contracting M_ab[c,d] = g_acbd over all (c, d).  The g+- of
// the pairs of a block of a come from the tensor-core GEMM G = L_block^T L (one K split, so each
// element is the same dot product whatever the block) and one pass that forms the sums and
// differences and writes them as planes (form_pm_planes).
//
// ladder_pairs fills mbuf with the planes of all pairs, P+ then P-.  Those of the untransformed L_vv
// (untransformed = true) stay valid until the Cholesky vectors change, so the mixed residual forms
// them once per Cholesky set; any other L_vv (T1-transformed, or transposed for the adjoint) is
// formed once per call and shared by all vectors of that call.
namespace {

struct PairShape {
    int64_t nvp, nvm;     // pairs c >= d, c > d (the K of the + and - GEMMs, and the pairs a >= b, a > b)
    int64_t kp, km;       // K padded
    int64_t rows_p, rows_m;   // rows of all pairs padded for the B operand
    size_t plane_p() const { return (size_t)rows_p * kp; }
    size_t plane_m() const { return (size_t)rows_m * km; }
};

PairShape pair_shape(int64_t nv) {
    PairShape p;
    p.nvp = nv * (nv + 1) / 2;
    p.nvm = nv * (nv - 1) / 2;
    p.kp = tc_pad_k(p.nvp);
    p.km = tc_pad_k(std::max<int64_t>(p.nvm, 1));
    p.rows_p = tc_pad_rows_b(p.nvp);
    p.rows_m = tc_pad_rows_b(std::max<int64_t>(p.nvm, 1));
    return p;
}

}  // namespace

// L_vv as (J, c, a): the columns (c, a) of one block of a are contiguous
DBuf Context::lvv_jca(const double *Lvv) {
    DBuf LT = dalloc(nJ * nv * nv, ex.stream);
    TV src = tv(Lvv, {nJ, nv, nv});   // [J, a, c]
    TV dst = tv(LT.d(), {nJ, nv, nv});
    dst.s[1] = nJ * nv;   // a
    dst.s[2] = nJ;        // c
    permute_add(ex, 1.0, src, 0.0, dst);
    return LT;
}

// g+- planes of the pairs a in [a0, a1) from LT = lvv_jca(L_vv): P+ rows a(a+1)/2 + b - rowp0 of a
// buffer of rows_p padded rows per plane, P- rows a(a-1)/2 + b - rowm0 (rows_m per plane); G holds at
// least n_v (a1 - a0) x n_v a1 doubles
void Context::form_pair_planes(const double *LT, int64_t a0, int64_t a1, double *G, __nv_bfloat16 *Pp,
                               int64_t rows_p, int64_t rowp0, __nv_bfloat16 *Pm, int64_t rows_m, int64_t rowm0) {
    const PairShape ps = pair_shape(nv);
    const int64_t M = nv * (a1 - a0), N = nv * a1;
    // G[(c, a), (d, b)] = sum_J L_ac L_bd
    mixed_gemm(ex, true, false, M, N, nJ, 1.0, LT + nJ * nv * a0, nJ, LT, nJ, 0.0, G, M, 1);
    form_pm_planes(ex, G, M, nv, a0, a1, ex.planes, Pp, ps.kp, (size_t)rows_p * ps.kp, rowp0, Pm, ps.km,
                   (size_t)rows_m * ps.km, rowm0);
    ex.flops += 2.0 * double(M) * double(N) * double(nJ);
}

// Whether the split-bf16 pair integrals of all pairs stay resident: they must fit the budget
// (ccsd_gpu_options.ladder_pair_budget, else half of the free device memory).  Otherwise the ladder
// forms them block by block in every call (ladder_tc_streamed), as eT's omega_ccsd_a2 does.
bool Context::ladder_pairs_resident() {
    const PairShape ps = pair_shape(nv);
    const double need = 2.0 * ex.planes * (double)(ps.plane_p() + ps.plane_m());
    if (ladder_pair_budget > 0) return need <= (double)ladder_pair_budget;
    if (mbuf_bytes >= need) return true;
    size_t free_b = 0, total_b = 0;
    CU_CHECK(cudaMemGetInfo(&free_b, &total_b));
    return need <= 0.5 * (double)free_b;
}

void Context::ladder_pairs(const double *Lvv, bool untransformed) {
    const int np = ex.planes;
    if (untransformed && mbuf_kind == 1 && mbuf_version == l_version && mbuf_planes == np) return;
    // a prepared transformation keeps the integrals of its (T1-transformed or transposed) vectors
    // for the next transformation of the same preparation
    if (!untransformed && pairs_reuse_id >= 0 && mbuf_kind == 2 && mbuf_reuse == pairs_reuse_id &&
        mbuf_src == Lvv && mbuf_version == l_version && mbuf_planes == np)
        return;
    cudaStream_t s = ex.stream;
    const PairShape ps = pair_shape(nv);
    const size_t bytes = sizeof(__nv_bfloat16) * np * (ps.plane_p() + ps.plane_m());
    // padding rows and K positions are never written and must read as zero; P- moves when the plane
    // count changes, so the buffer is cleared then too
    if (mbuf_bytes < bytes) {
        mbuf = DBuf(bytes, s);
        mbuf_bytes = mbuf.bytes();
        CU_CHECK(cudaMemsetAsync(mbuf.as<void>(), 0, mbuf_bytes, s));
    } else if (mbuf_planes != np) {
        CU_CHECK(cudaMemsetAsync(mbuf.as<void>(), 0, mbuf_bytes, s));
    }
    __nv_bfloat16 *Pp = mbuf.as<__nv_bfloat16>(), *Pm = Pp + np * ps.plane_p();
    DBuf LT = lvv_jca(Lvv);
    // blocks of a whose G fits in about 2 GB
    const int64_t nA = ladder_batch > 0 ? ladder_batch
                                        : std::max<int64_t>(1, std::min<int64_t>(nv, (int64_t)(2.0e9 / (8.0 * nv * nv * nv))));
    DBuf G = dalloc(nv * std::min(nA, nv) * nv * nv, s);
    for (int64_t a0 = 0; a0 < nv; a0 += nA)
        form_pair_planes(LT.d(), a0, std::min(nv, a0 + nA), G.d(), Pp, ps.rows_p, 0, Pm, ps.rows_m, 0);
    mbuf_kind = untransformed ? 1 : 2;
    mbuf_version = l_version;
    mbuf_planes = np;
    mbuf_src = untransformed ? nullptr : Lvv;
    mbuf_reuse = untransformed ? -1 : pairs_reuse_id;
    cache_epoch++;
}

// t+ and t- planes of nvec packed vectors (the A operands of the +/- GEMMs)
Context::TPlanes Context::t_planes(const double *t2, int64_t nvec) {
    const PairShape ps = pair_shape(nv);
    const int np = ex.planes;
    const int64_t nop = no * (no + 1) / 2, nom = no * (no - 1) / 2;
    TPlanes T;
    T.rows_p = tc_pad_rows_a(nvec * nop);
    T.rows_m = tc_pad_rows_a(std::max<int64_t>(nvec * nom, 1));
    T.p = DBuf(sizeof(__nv_bfloat16) * np * T.rows_p * ps.kp, ex.stream);
    T.m = DBuf(sizeof(__nv_bfloat16) * np * T.rows_m * ps.km, ex.stream);
    build_tpm_planes(ex, t2, nvec, no, nv, true, T.rows_p, ps.kp, np, T.p.as<__nv_bfloat16>());
    build_tpm_planes(ex, t2, nvec, no, nv, false, T.rows_m, ps.km, np, T.m.as<__nv_bfloat16>());
    return T;
}

// om2[v] += the ladder of the pairs a in [a0, a1), whose g+- planes are Pp / Pm (row 0 = the
// block's first pair, prow / mrow padded rows per plane)
void Context::ladder_pm_block(const TPlanes &T, int64_t nvec, const __nv_bfloat16 *Pp, int64_t prow,
                              const __nv_bfloat16 *Pm, int64_t mrow, int64_t a0, int64_t a1, double *om2) {
    const PairShape ps = pair_shape(nv);
    const int64_t nop = no * (no + 1) / 2, nom = no * (no - 1) / 2;
    const int64_t nabp = a1 * (a1 + 1) / 2 - a0 * (a0 + 1) / 2, nabm = a1 * (a1 - 1) / 2 - a0 * (a0 - 1) / 2;
    const int64_t ldp = nvec * nop, ldm = std::max<int64_t>(nvec * nom, 1);
    DBuf wp = dalloc(ldp * nabp, ex.stream), wm = dalloc(ldm * std::max<int64_t>(nabm, 1), ex.stream);
    tc_gemm_f64(ex, T.p.as<__nv_bfloat16>(), T.rows_p, Pp, prow, ps.kp, ldp, nabp, ps.nvp, 0.5, 0.0, wp.d(), ldp, 1);
    if (nom > 0 && nabm > 0)
        tc_gemm_f64(ex, T.m.as<__nv_bfloat16>(), T.rows_m, Pm, mrow, ps.km, nvec * nom, nabm, ps.nvm, 0.5, 0.0, wm.d(),
                    ldm, 1);
    for (int64_t v = 0; v < nvec; v++)
        add_omega_pm(ex, om2 + v * nt2, wp.d() + v * nop, wm.d() + v * nom, no, nv, a0, a1, ldp, ldm);
    ex.flops += 2.0 * double(ldp) * double(nabp) * double(ps.nvp) + 2.0 * double(nvec * nom) * double(nabm) * double(ps.nvm);
}

void Context::ladder_tc(const double *Lvv, const double *t2, double *om2, int64_t nvec, bool untransformed) {
    if (!ladder_pairs_resident()) {
        if (mbuf) {
            mbuf.release();
            mbuf_bytes = 0;
            mbuf_kind = 0;
            cache_epoch++;
        }
        ladder_tc_streamed(Lvv, t2, om2, nvec);
        return;
    }
    ladder_pairs(Lvv, untransformed);
    const PairShape ps = pair_shape(nv);
    const TPlanes T = t_planes(t2, nvec);
    const __nv_bfloat16 *Pp = mbuf.as<__nv_bfloat16>(), *Pm = Pp + ex.planes * ps.plane_p();
    ladder_pm_block(T, nvec, Pp, ps.rows_p, Pm, ps.rows_m, 0, nv, om2);
}

// The same ladder with bounded memory: the g+- planes of a block of consecutive a are formed into
// one buffer and contracted right away (omega_ccsd_a2's (a, b) batching on the tensor cores,
// omega_ccsd.F90:236-458).  Every output element is the dot product it is in the resident form (the
// same planes, one K split, the same K chunks), so the result equals the resident ladder's bit for bit.
void Context::ladder_tc_streamed(const double *Lvv, const double *t2, double *om2, int64_t nvec) {
    cudaStream_t s = ex.stream;
    const int np = ex.planes;
    const PairShape ps = pair_shape(nv);
    const int64_t nop = no * (no + 1) / 2, nom = no * (no - 1) / 2;
    const int64_t ldp = nvec * nop, ldm = std::max<int64_t>(nvec * nom, 1);
    DBuf LT = lvv_jca(Lvv);
    const TPlanes T = t_planes(t2, nvec);
    // blocks: consecutive a whose G, planes and W fit the budget (or a quarter of the free memory),
    // at least one a each
    int64_t budget = ladder_pair_budget;
    if (budget <= 0) {
        size_t free_b = 0, total_b = 0;
        CU_CHECK(cudaMemGetInfo(&free_b, &total_b));
        budget = (int64_t)(0.25 * (double)free_b);
    }
    auto block_bytes = [&](int64_t a0, int64_t a1) {
        const int64_t nabp = a1 * (a1 + 1) / 2 - a0 * (a0 + 1) / 2, nabm = a1 * (a1 - 1) / 2 - a0 * (a0 - 1) / 2;
        return 8.0 * double(nv * (a1 - a0)) * double(nv * a1) +
               2.0 * np * (double(tc_pad_rows_b(nabp)) * ps.kp + double(tc_pad_rows_b(std::max<int64_t>(nabm, 1))) * ps.km) +
               8.0 * (double(ldp) * nabp + double(ldm) * nabm);
    };
    std::vector<std::pair<int64_t, int64_t>> blocks;
    int64_t g_max = 0, prow_max = 0, mrow_max = 0;
    for (int64_t a0 = 0; a0 < nv;) {
        int64_t a1 = a0 + 1;
        while (a1 < nv && block_bytes(a0, a1 + 1) <= (double)budget) a1++;
        blocks.emplace_back(a0, a1);
        g_max = std::max(g_max, nv * (a1 - a0) * nv * a1);
        prow_max = std::max(prow_max, tc_pad_rows_b(a1 * (a1 + 1) / 2 - a0 * (a0 + 1) / 2));
        mrow_max = std::max(mrow_max, tc_pad_rows_b(std::max<int64_t>(a1 * (a1 - 1) / 2 - a0 * (a0 - 1) / 2, 1)));
        a0 = a1;
    }
    DBuf G = dalloc(g_max, s);
    DBuf P(sizeof(__nv_bfloat16) * np * (size_t(prow_max) * ps.kp + size_t(mrow_max) * ps.km), s);
    // K positions beyond the pair count are never written and must read as zero
    CU_CHECK(cudaMemsetAsync(P.as<void>(), 0, P.bytes(), s));
    __nv_bfloat16 *Pp = P.as<__nv_bfloat16>(), *Pm = Pp + np * size_t(prow_max) * ps.kp;
    for (const auto &blk : blocks) {
        const int64_t a0 = blk.first, a1 = blk.second;
        form_pair_planes(LT.d(), a0, a1, G.d(), Pp, prow_max, a0 * (a0 + 1) / 2, Pm, mrow_max,
                         std::max<int64_t>(a0 * (a0 - 1) / 2, 0));
        ladder_pm_block(T, nvec, Pp, prow_max, Pm, mrow_max, a0, a1, om2);
    }
}

// Mixed precision keeps the ovvv integrals of the untransformed Cholesky vectors resident as split
// bf16, ybuf[plane][k + no*b][c + nv*d] = g_kcbd (o v^3 elements per plane: 4.2 GB for both planes
// at o = 32, v = 320), formed once per Cholesky set by one tensor-core GEMM whose epilogue writes
// the planes.  The ladder's Y intermediates then cost one GEMM of o^2 x o v x v^2 per call instead
// of re-forming g_kcbd in batches (and permuting and splitting it) every time.
bool Context::ovvv_resident() {
    const size_t need = sizeof(__nv_bfloat16) * (size_t)ex.planes * (size_t)tc_pad_rows_a(nov) * tc_pad_k(nv * nv);
    if (ybuf_bytes >= need) return true;
    if (ybuf_fit < 0 || ybuf_fit_version != l_version || ybuf_fit_planes != ex.planes) {
        size_t free_b = 0, total_b = 0;
        CU_CHECK(cudaMemGetInfo(&free_b, &total_b));
        ybuf_fit = need < free_b / 4 ? 1 : 0;
        ybuf_fit_version = l_version;
        ybuf_fit_planes = ex.planes;
    }
    return ybuf_fit == 1;
}

void Context::ovvv_pairs() {
    const int np = ex.planes;
    if (ybuf_version == l_version && ybuf_planes == np) return;
    cudaStream_t s = ex.stream;
    const int64_t nv2 = nv * nv, Jp = tc_pad_k(nJ), Kq = tc_pad_k(nv2);
    // L_ov split rows c + nv*k: L_ov[J, k, c] sits at J + nJ*(k + no*c); copy to (J, c, k) first
    const int64_t o_rows = tc_pad_rows_a(nov);
    DBuf LOS(sizeof(__nv_bfloat16) * np * o_rows * Jp, s);
    {
        DBuf LO = dalloc(nJ * nov, s);
        TV dst = tv(LO.d(), {nJ, no, nv});   // [J, k, c] at J + nJ*(c + nv*k)
        dst.s[1] = nJ * nv;
        dst.s[2] = nJ;
        permute_add(ex, 1.0, tv(L_ov.d(), {nJ, no, nv}), 0.0, dst);
        split_rows(ex, LO.d(), nJ, 1, nov, nJ, o_rows, Jp, LOS.as<__nv_bfloat16>());
    }
    // L_vv split rows d + nv*b: L_vv[J, b, d] sits at J + nJ*(b + nv*d); copy to (J, d, b)
    const int64_t v_rows = tc_pad_rows_b(nv2);
    DBuf LVS(sizeof(__nv_bfloat16) * np * v_rows * Jp, s);
    {
        DBuf LV = dalloc(nJ * nv2, s);
        TV dst = tv(LV.d(), {nJ, nv, nv});   // [J, b, d] at J + nJ*(d + nv*b)
        dst.s[1] = nJ * nv;
        dst.s[2] = nJ;
        permute_add(ex, 1.0, tv(L_vv.d(), {nJ, nv, nv}), 0.0, dst);
        split_rows(ex, LV.d(), nJ, 1, nv2, nJ, v_rows, Jp, LVS.as<__nv_bfloat16>());
    }
    const int64_t yrows = tc_pad_rows_a(nov);
    const size_t need = sizeof(__nv_bfloat16) * (size_t)np * (size_t)yrows * Kq;
    if (ybuf_bytes < need) {
        ybuf = DBuf();
        ybuf = DBuf(need, s);
        ybuf_bytes = need;
        // padding rows and K positions are never written and must read as zero
        CU_CHECK(cudaMemsetAsync(ybuf.as<void>(), 0, need, s));
    }
    tc_gemm_ovvv(ex, LOS.as<__nv_bfloat16>(), o_rows, LVS.as<__nv_bfloat16>(), v_rows, Jp, no, nv,
                 ybuf.as<__nv_bfloat16>(), yrows, Kq, nJ);
    ybuf_version = l_version;
    ybuf_planes = np;
    cache_epoch++;
}

void Context::ladder_y0(const double *tf, double *Y) {
    ovvv_pairs();
    cudaStream_t s = ex.stream;
    const int64_t nv2 = nv * nv, oo = no * no, Kq = tc_pad_k(nv2), yrows = tc_pad_rows_a(nov);
    const int64_t rows_T = tc_pad_rows_b(oo);
    DBuf TS(sizeof(__nv_bfloat16) * ex.planes * rows_T * Kq, s);
    {
        // tau split rows i + no*j, K position c + nv*d: copy tau[c, i, d, j] to (c, d, i, j)
        DBuf TT = dalloc(oo * nv2, s);
        TV dst = tv(TT.d(), {nv, no, nv, no});
        dst.s[1] = nv2;        // i
        dst.s[2] = nv;         // d
        dst.s[3] = nv2 * no;   // j
        permute_add(ex, 1.0, tv(tf, {nv, no, nv, no}), 0.0, dst);
        split_rows(ex, TT.d(), nv2, 1, oo, nv2, rows_T, Kq, TS.as<__nv_bfloat16>());
    }
    // Yt[(k + no*b) + nov*(i + no*j)], then Y[k, i, b, j]
    DBuf Yt = dalloc(nov * oo, s);
    tc_gemm_f64_tuned(ex, ybuf.as<__nv_bfloat16>(), yrows, TS.as<__nv_bfloat16>(), rows_T, Kq, nov, oo, nv2, 1.0, 0.0,
                      Yt.d(), nov, 0);
    TV src = tv(Yt.d(), {no, no, nv, no});   // (k, i, b, j)
    src.s[1] = nov;
    src.s[2] = no;
    src.s[3] = nov * no;
    permute_add(ex, 1.0, src, 0.0, tv(Y, {no, no, nv, no}));
}

void Context::ladder_y_t1(const double *t1, const double *Ltvv, const double *tf, double *Y) {
    if (ex.prec == Prec::MIXED && ovvv_resident()) {
        ladder_y0(tf, Y);
    } else if (ex.prec != Prec::MIXED && f64_resident()) {
        f64_integrals();
        contract(ex, "kbcd,cidj->kibj", 1.0, tv(f64_ovvv.d(), {no, nv, nv, nv}), tv(tf, {nv, no, nv, no}), 0.0,
                 tv(Y, {no, no, nv, no}));
    } else {
        ladder_y(Ltvv, tf, Y);
        return;
    }
    // L~_bd = L_bd - sum_l t_bl L_ld, so g_kc~bd = g_kcbd - sum_l t_bl g_kcld
    DBuf Q = dalloc(no * no * no * no, ex.stream);
    contract(ex, "kcld,cidj->kilj", 1.0, tv(g_ovov_const(), {no, nv, no, nv}), tv(tf, {nv, no, nv, no}), 0.0,
             tv(Q.d(), {no, no, no, no}));
    contract(ex, "bl,kilj->kibj", -1.0, tv(t1, {nv, no}), tv(Q.d(), {no, no, no, no}), 1.0,
             tv(Y, {no, no, nv, no}));
}

// The A2 ladder of the residual on the tensor cores, without forming T1-transformed integrals.
// With L~_vv = L_vv - t1 L_ov (the T1 transformation of the vv block),
//   g~_acbd = g_acbd - sum_k t_ak g_kcbd - sum_l t_bl g_acld + sum_kl t_ak t_bl g_kcld,
// so X_aibj = sum_cd g~_acbd t_cidj (symmetric in ai <-> bj) is
//   X = sum_cd g_acbd t_cidj - (A + A^T) + T4,   A_aibj = sum_k t_ak Y_kibj,
//   Y_kibj = sum_cd g_kcbd t_cidj,   T4_aibj = sum_kl t_ak t_bl Q_kilj,   Q_kilj = sum_cd g_kcld t_cidj,
// (the A^T term uses sum_cd g_acld t_cidj = Y_ljai), all with untransformed integrals: the v^4
// integrals are formed once per Cholesky set instead of every iteration, the corrections cost
// o^2 v^3 N_J + o^3 v^3.  The ladder adds pack(X) with the doubles diagonal halved to om2.
void Context::ladder_residual_mixed(const double *t1, const double *tf, const double *t2, double *om2) {
    cudaStream_t s = ex.stream;
    ladder_tc(L_vv.d(), t2, om2, 1, true);
    DBuf Y = dalloc(no * no * nv * no, s);
    if (ovvv_resident()) ladder_y0(tf, Y.d());
    else ladder_y(L_vv.d(), tf, Y.d());
    ladder_t1_corrections(t1, tf, Y.d(), om2);
}

void Context::ladder_t1_corrections(const double *t1, const double *tf, const double *Y0, double *om2) {
    cudaStream_t s = ex.stream;
    // the terms below are A_aibj (not symmetric); omega gets pack(A + A^T) with the diagonal halved
    DBuf A = dalloc(nov * nov, s);
    contract(ex, "ak,kibj->aibj", -1.0, tv(t1, {nv, no}), tv(Y0, {no, no, nv, no}), 0.0,
             tv(A.d(), {nv, no, nv, no}));
    {
        DBuf Q = dalloc(no * no * no * no, s), B = dalloc(nv * no * no * no, s);
        contract(ex, "kcld,cidj->kilj", 1.0, tv(g_ovov_const(), {no, nv, no, nv}), tv(tf, {nv, no, nv, no}), 0.0,
                 tv(Q.d(), {no, no, no, no}));
        contract(ex, "ak,kilj->ailj", 1.0, tv(t1, {nv, no}), tv(Q.d(), {no, no, no, no}), 0.0,
                 tv(B.d(), {nv, no, no, no}));
        // the symmetric term sum_l t_bl B_ailj enters at half weight (pack(A + A^T) adds it twice), in
        // its mirrored form sum_l t_al B_bjli, whose output index order (a | i, b, j) lies in A's own
        // layout, so the product writes A in place instead of through a reordered copy
        contract(ex, "al,bjli->aibj", 0.5, tv(t1, {nv, no}), tv(B.d(), {nv, no, no, no}), 1.0,
                 tv(A.d(), {nv, no, nv, no}));
    }
    pack_sym_add(ex, A.d(), om2, nov);
}

// FP64 integrals of the untransformed vectors, resident while they fit in half of the free memory
// (50 GB at o = 32, v = 320): the +/- ladder integrals of all pairs (eT's packing, formed block by
// block exactly as the per-call ladder forms them) and g_kcbd.
bool Context::f64_resident() {
    if (!f64_resident_on) return false;
    if (f64_version == l_version) return true;
    const int64_t nvp = nv * (nv + 1) / 2, nvm = nv * (nv - 1) / 2;
    // buffers of this shape already held (integrals of earlier Cholesky vectors) are reused
    if (f64_gp.bytes() == sizeof(double) * nvp * nvp && f64_ovvv.bytes() == sizeof(double) * nov * nv * nv)
        return true;
    if (f64_fit < 0 || f64_fit_version != l_version) {
        const double need = 8.0 * (double(nvp) * nvp + double(nvm) * nvm + double(nov) * nv * nv);
        size_t free_b = 0, total_b = 0;
        CU_CHECK(cudaMemGetInfo(&free_b, &total_b));
        f64_fit = need < 0.5 * double(free_b) ? 1 : 0;
        f64_fit_version = l_version;
    }
    return f64_fit == 1;
}

void Context::f64_integrals() {
    if (f64_version == l_version) return;
    cudaStream_t s = ex.stream;
    const Prec keep = ex.prec;
    ex.prec = Prec::FP64;
    const int64_t nvp = nv * (nv + 1) / 2, nvm = nv * (nv - 1) / 2;
    auto hold = [&](DBuf &b, int64_t n) {
        if (b.bytes() == sizeof(double) * (size_t)n) return;
        b = DBuf();
        b = dalloc(n, s);
    };
    hold(f64_gp, nvp * nvp);
    hold(f64_gm, std::max<int64_t>(nvm * nvm, 1));
    hold(f64_ovvv, nov * nv * nv);
    {
        // L_vv as (J, c, a): columns (c, a) of one a-block are contiguous
        DBuf LT = dalloc(nJ * nv * nv, s);
        TV dst = tv(LT.d(), {nJ, nv, nv});
        dst.s[1] = nJ * nv;
        dst.s[2] = nJ;
        permute_add(ex, 1.0, tv(L_vv.d(), {nJ, nv, nv}), 0.0, dst);
        const int64_t nA = std::max<int64_t>(1, std::min<int64_t>(nv, (int64_t)(4.0e9 / (8.0 * nv * nv * nv))));
        DBuf G = dalloc(nv * nA * nv * nv, s);
        for (int64_t a0 = 0; a0 < nv; a0 += nA) {
            const int64_t a1 = std::min(nv, a0 + nA), M = nv * (a1 - a0), N = nv * a1;
            gemm(ex, true, false, M, N, nJ, 1.0, LT.d() + nJ * nv * a0, nJ, LT.d(), nJ, 0.0, G.d(), M);
            form_gpm(ex, G.d(), M, f64_gp.d() + nvp * (a0 * (a0 + 1) / 2),
                     f64_gm.d() + nvm * std::max<int64_t>(a0 * (a0 - 1) / 2, 0), nv, a0, a1);
        }
    }
    // g_kcbd as [k, b, c, d]
    contract(ex, "Jkc,Jbd->kbcd", 1.0, tv(L_ov.d(), {nJ, no, nv}), tv(L_vv.d(), {nJ, nv, nv}), 0.0,
             tv(f64_ovvv.d(), {no, nv, nv, nv}));
    ex.prec = keep;
    f64_version = l_version;
    cache_epoch++;
}

int Context::f64_digit_planes(int digits) {
    if (f64_dig_version == f64_version && f64_dig_digits == digits) return f64_dig_level;
    const int64_t nvp = nv * (nv + 1) / 2, nvm = nv * (nv - 1) / 2;
    auto planes = [&](int64_t rows, int64_t k) {
        return (double)digits * (double)((rows + 127) / 128 * 128) * (double)((k + 63) / 64 * 64);
    };
    const double ladder = planes(nvp, nvp) + (nvm > 0 ? planes(nvm, nvm) : 0.0), ovvv = planes(nov, nv * nv);
    for (OzPlanes *p : {&f64_gp_dig, &f64_gm_dig, &f64_ovvv_dig}) p->buf.release();
    size_t free_b = 0, total_b = 0;
    CU_CHECK(cudaMemGetInfo(&free_b, &total_b));
    const double room = 0.6 * (double)free_b;
    f64_dig_level = ladder + ovvv <= room ? 2 : ladder <= room ? 1 : 0;
    if (f64_dig_level >= 1) {
        ozaki_prepare(ex, true, nvp, nvp, f64_gp.d(), nvp, digits, f64_gp_dig);
        if (nvm > 0) ozaki_prepare(ex, true, nvm, nvm, f64_gm.d(), nvm, digits, f64_gm_dig);
    }
    if (f64_dig_level == 2) ozaki_prepare(ex, false, nov, nv * nv, f64_ovvv.d(), nov, digits, f64_ovvv_dig);
    f64_dig_version = f64_version;
    f64_dig_digits = digits;
    cache_epoch++;
    return f64_dig_level;
}

void Context::ladder_residual_f64(const double *t1, const double *tf, const double *t2, double *om2) {
    f64_integrals();
    cudaStream_t s = ex.stream;
    const int64_t nop = no * (no + 1) / 2, nom = no * (no - 1) / 2;
    const int64_t nvp = nv * (nv + 1) / 2, nvm = nv * (nv - 1) / 2;
    const int64_t ldm = std::max<int64_t>(nom, 1);
    // on the digit GEMM the constant operands come as digit planes kept per Cholesky set (products
    // big enough for it, as gemm() decides)
    const int digits = ex.fp64_digits;
    const bool big = digits > 0 && 2.0 * double(nop) * double(nvp) * double(nvp) >= ex.fp64_digits_min_flops &&
                     (ex.fp64_digits_min_flops <= 1 || (nop >= 256 && nvp >= 256));
    const int level = big ? f64_digit_planes(digits) : 0;
    // X0 = sum_cd g_acbd t_cidj of the untransformed integrals, all pairs in two GEMMs
    {
        DBuf tp = dalloc(nop * nvp, s), tm = dalloc(ldm * std::max<int64_t>(nvm, 1), s);
        build_tpm(ex, t2, tp.d(), tm.d(), no, nv, nop, ldm);
        DBuf wp = dalloc(nop * nvp, s), wm = dalloc(ldm * std::max<int64_t>(nvm, 1), s);
        if (level >= 1) {
            ozaki_gemm(ex, false, false, nop, nvp, nvp, 0.5, tp.d(), nop, f64_gp.d(), nvp, 0.0, wp.d(), nop, digits,
                       nullptr, &f64_gp_dig);
            if (nom > 0 && nvm > 0)
                ozaki_gemm(ex, false, false, nom, nvm, nvm, 0.5, tm.d(), ldm, f64_gm.d(), nvm, 0.0, wm.d(), ldm,
                           digits, nullptr, &f64_gm_dig);
            ex.flops += 2.0 * (double(nop) * nvp * nvp + double(nom) * nvm * nvm);
        } else {
            gemm(ex, false, false, nop, nvp, nvp, 0.5, tp.d(), nop, f64_gp.d(), nvp, 0.0, wp.d(), nop, false);
            if (nom > 0 && nvm > 0)
                gemm(ex, false, false, nom, nvm, nvm, 0.5, tm.d(), ldm, f64_gm.d(), nvm, 0.0, wm.d(), ldm, false);
        }
        add_omega_pm(ex, om2, wp.d(), wm.d(), no, nv, 0, nv, nop, ldm);
    }
    DBuf Y = dalloc(no * no * nv * no, s);
    if (level == 2) {
        // Y_kibj = sum_cd g_kbcd t_cidj: t as [(c, d), (i, j)], the product [(k, b), (i, j)], then Y
        DBuf TT = dalloc(nv * nv * no * no, s), W = dalloc(nov * no * no, s);
        TV tt = tv(TT.d(), {nv, no, nv, no});   // (c, i, d, j) at c + nv d + nv^2 (i + no j)
        tt.s[1] = nv * nv;
        tt.s[2] = nv;
        tt.s[3] = nv * nv * no;
        permute_add(ex, 1.0, tv(tf, {nv, no, nv, no}), 0.0, tt);
        ozaki_gemm(ex, false, false, nov, no * no, nv * nv, 1.0, f64_ovvv.d(), nov, TT.d(), nv * nv, 0.0, W.d(), nov,
                   digits, &f64_ovvv_dig, nullptr);
        ex.flops += 2.0 * double(nov) * double(no * no) * double(nv * nv);
        TV w = tv(W.d(), {no, no, nv, no});     // (k, i, b, j) at k + no b + no nv (i + no j)
        w.s[1] = no * nv;
        w.s[2] = no;
        w.s[3] = no * nv * no;
        permute_add(ex, 1.0, w, 0.0, tv(Y.d(), {no, no, nv, no}));
    } else {
        contract(ex, "kbcd,cidj->kibj", 1.0, tv(f64_ovvv.d(), {no, nv, nv, nv}), tv(tf, {nv, no, nv, no}), 0.0,
                 tv(Y.d(), {no, no, nv, no}));
    }
    ladder_t1_corrections(t1, tf, Y.d(), om2);
}

// ---------------------------------------------------------------------------
// run_diis_cc_gs (src/solvers/cc/diis_cc_gs_class.F90:209-315)
// ---------------------------------------------------------------------------
int Context::solve_gs(const ccsd_gpu_solver_options *o, double *energy_out, int32_t *iters, double *history) {
    REQUIRE(have_t && have_L && have_h, CCSD_GPU_ESTATE, "inputs/amplitudes not set");
    const int maxit = o && o->max_iterations > 0 ? o->max_iterations : 100;
    const int dim = o && o->diis_dimension > 0 ? std::min(o->diis_dimension, 16) : 8;
    const double othr = o && o->omega_threshold > 0 ? o->omega_threshold : 1e-5;
    const double ethr = o ? o->energy_threshold : 1e-5;
    const double refine = o && o->refine_threshold > 0 ? o->refine_threshold : 1e-4;
    const double rtarget = o && o->refine_target > 0 ? o->refine_target : othr;
    const int rdig = o ? o->refresh_digits : 0;
    REQUIRE(rdig == 0 || rdig == -1 || (rdig >= 4 && rdig <= 7), CCSD_GPU_EINVAL,
            "refresh_digits must be 0 (default), -1 (DGEMM) or 4..7");
    // arithmetic of the FP64 evaluations: the option, else the context's setting (ccsd_gpu_set_fp64_digits)
    const int user_digits = ex.fp64_digits;
    const int fp64_digits = rdig > 0 ? rdig : (rdig < 0 ? 0 : user_digits);
    cudaStream_t s = ex.stream;
    const auto trace_t0 = std::chrono::steady_clock::now();
    orbital_differences(ex, eps.d(), no, nv, epsdiff.d());
    DBuf omega_v = dalloc(namp, s);
    std::vector<DBuf> errs(dim), pars(dim);
    for (int k = 0; k < dim; k++) {
        errs[k] = dalloc(namp, s);
        pars[k] = dalloc(namp, s);
    }
    DBuf Gs = dalloc(16 * 16, s), dots = dalloc(16, s), wts = dalloc(16, s);
    DBuf stat(sizeof(int), s);
    std::vector<int> order;   // slots, oldest first
    const Prec user = ex.prec;
    const bool mixed = (user == Prec::MIXED);
    // the arithmetic changes during the solve; the caller's choice is restored on every exit
    struct Restore {
        Exec &ex;
        Prec prec;
        int planes, digits;
        ~Restore() {
            ex.prec = prec;
            ex.planes = planes;
            ex.fp64_digits = digits;
        }
    } restore{ex, ex.prec, ex.planes, ex.fp64_digits};
    // Mixed precision with defect correction: Omega~(t) = Omega_mixed(t) + c, where
    // c = Omega_fp64(t_c) - Omega_mixed(t_c) is refreshed by one FP64 evaluation at a time.  The mixed
    // error d(t) = Omega_fp64(t) - Omega_mixed(t) is mostly frozen, but the truncating FP32
    // accumulation of the tensor cores rounds differently as soon as t changes, so d drifts even for
    // tiny steps (a 1e-10 step moves it by ~2e-9, a long solve path by ~4e-7 at o=32, v=320):
    // iterating on Omega~ lowers the true residual only down to that drift.  The policy:
    //  * first refresh when |Omega_mixed| < refine_threshold;
    //  * refresh again when |Omega~| meets the convergence test (the refresh is then the FP64
    //    convergence check), when it stops falling (no 30% reduction in three iterations), or, if
    //    the expected drift is above refine_target (default: the residual threshold), once |Omega~|
    //    is below half of it
    //    (further mixed iterations would not lower the true residual).  The expected drift is what
    //    the previous refresh measured; after the first refresh, which measures the whole mixed
    //    error d rather than its drift, it is 0.15 |d| (the ratio seen along bf16x3 solve paths);
    //  * a refresh that finds the residual function moved by more than 0.3 of a true residual still
    //    above refine_target (drift dominates), or a cycle that gained less than a factor 2, hands
    //    the remaining iterations to FP64.
    // A refresh changes the residual function by the same vector c_new - c_old at every t (up to the
    // drift), so the stored DIIS error vectors are shifted by its quasi-Newton image (and their Gram
    // matrix recomputed) instead of restarting the DIIS subspace.
    DBuf om_mixed = mixed ? dalloc(namp, s) : DBuf(), corr = mixed ? dalloc(namp, s) : DBuf();
    DBuf moved_v = mixed ? dalloc(namp, s) : DBuf();
    bool have_corr = false;
    double r_c = 0.0, drift_est = 0.0;
    double prev = 0.0, e = 0.0;
    int it = 0;
    bool conv = false;
    auto norm_of = [&](const double *v) {
        dot(ex, v, v, namp, scal.d());
        double nrm2;
        CU_CHECK(cudaMemcpyAsync(&nrm2, scal.d(), sizeof(double), cudaMemcpyDeviceToHost, s));
        CU_CHECK(cudaStreamSynchronize(s));
        return std::sqrt(nrm2);
    };
    bool reset_diis = false, fp64_final = false;
    int last_check = 0;
    std::vector<double> norms;
    // CCSD_GPU_TRACE=1: one line per iteration on stderr with the refinement decisions
    const bool trace = std::getenv("CCSD_GPU_TRACE") && std::atoi(std::getenv("CCSD_GPU_TRACE")) >= 1;
    auto trace_ms = [&]() {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - trace_t0).count();
    };
    // the stream-ordered pool's reserved and used memory (GB), printed with each traced iteration
    auto trace_pool = [&](double &reserved, double &used) {
        reserved = used = 0.0;
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) return;
        uint64_t r = 0, u = 0;
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r);
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u);
        reserved = 1e-9 * (double)r;
        used = 1e-9 * (double)u;
    };
    double trace_moved = 0.0;
    const char *trace_why = "";
    if (trace) {
        CU_CHECK(cudaStreamSynchronize(s));
        std::fprintf(stderr, "ccsd_gpu gs set-up (records allocated) t %.1f ms\n", trace_ms());
    }
    // shift every stored DIIS error vector by v and rebuild their Gram matrix
    auto shift_diis = [&](const double *v) {
        const int n = (int)order.size();
        if (n == 0) return;
        for (int k = 0; k < n; k++) axpby(ex, namp, 1.0, v, 1.0, errs[order[k]].d());
        std::vector<const double *> ptr(n);
        for (int k = 0; k < n; k++) ptr[k] = errs[order[k]].d();
        DBuf g = dalloc(16 * 16, s);
        for (int k = 0; k < n; k++) multi_dot(ex, ptr[k], ptr.data(), n, namp, g.d() + 16 * k);
        std::vector<double> gh(16 * 16), G(16 * 16, 0.0);
        CU_CHECK(cudaMemcpyAsync(gh.data(), g.d(), sizeof(double) * 256, cudaMemcpyDeviceToHost, s));
        CU_CHECK(cudaMemcpyAsync(G.data(), Gs.d(), sizeof(double) * 256, cudaMemcpyDeviceToHost, s));
        CU_CHECK(cudaStreamSynchronize(s));
        for (int a = 0; a < n; a++)
            for (int b = 0; b < n; b++) G[order[a] * 16 + order[b]] = gh[16 * a + b];
        CU_CHECK(cudaMemcpyAsync(Gs.d(), G.data(), sizeof(double) * 256, cudaMemcpyHostToDevice, s));
    };
    // FP64 Omega at the current t into omega_v (which holds Omega~ on entry); the correction becomes
    // Omega_fp64 - Omega_mixed
    auto fp64_check = [&]() {
        last_check = it;
        CU_CHECK(cudaMemcpyAsync(moved_v.d(), omega_v.d(), sizeof(double) * namp, cudaMemcpyDeviceToDevice, s));
        ex.prec = Prec::FP64;
        ex.fp64_digits = fp64_digits;
        omega(omega_v.d());
        ex.fp64_digits = user_digits;
        ex.prec = user;
        CU_CHECK(cudaMemcpyAsync(corr.d(), omega_v.d(), sizeof(double) * namp, cudaMemcpyDeviceToDevice, s));
        axpby(ex, namp, -1.0, om_mixed.d(), 1.0, corr.d());
        axpby(ex, namp, 1.0, omega_v.d(), -1.0, moved_v.d());   // c_new - c_old
        const double moved = norm_of(moved_v.d()), nrm64 = norm_of(omega_v.d());
        trace_moved = moved;
        drift_est = have_corr ? moved : 0.15 * moved;
        if (have_corr && ((moved > 0.3 * nrm64 && nrm64 >= rtarget) || nrm64 > 0.5 * r_c)) fp64_final = true;
        if (fp64_final) {
            reset_diis = true;
        } else {
            qn_precondition(ex, moved_v.d(), epsdiff.d(), namp, nt1);
            shift_diis(moved_v.d());
        }
        r_c = nrm64;
        have_corr = true;
        return nrm64;
    };
    double t_norm_done = 0.0, t_energy = 0.0, t_update = 0.0;
    while (it < maxit) {
        it++;
        const double t_start = trace ? trace_ms() : 0.0;
        refresh();
        e = energy();
        if (trace) t_energy = trace_ms() - t_start;
        double nrm;
        bool exact = !mixed;
        if (!mixed || fp64_final) {
            exact = true;
            if (fp64_final) {
                ex.prec = Prec::FP64;
                ex.fp64_digits = fp64_digits;
            }
            omega(omega_v.d());
            ex.fp64_digits = user_digits;
            ex.prec = user;
            nrm = norm_of(omega_v.d());
        } else {
            omega(om_mixed.d());
            CU_CHECK(cudaMemcpyAsync(omega_v.d(), om_mixed.d(), sizeof(double) * namp, cudaMemcpyDeviceToDevice, s));
            if (have_corr) axpby(ex, namp, 1.0, corr.d(), 1.0, omega_v.d());
            nrm = norm_of(omega_v.d());
            const bool econv0 = ethr < 0 || std::fabs(e - prev) < ethr;
            const bool stalled = it - last_check > 3 && norms.size() >= 3 && nrm > 0.7 * norms[norms.size() - 3];
            const bool below = have_corr && drift_est > rtarget && nrm < 0.5 * drift_est;
            trace_moved = 0.0;
            trace_why = "";
            if ((!have_corr && nrm < refine) || (nrm < othr && econv0) || below || stalled) {
                trace_why = !have_corr ? "refine" : (nrm < othr && econv0) ? "check" : below ? "cycle" : "stall";
                if (trace) std::fprintf(stderr, "ccsd_gpu gs %3d  mixed |Omega~| %.3e\n", it, nrm);
                nrm = fp64_check();
                exact = true;
            }
        }
        if (trace) {
            double pool_r, pool_u;
            trace_pool(pool_r, pool_u);
            // phases (host time between the solver's synchronisation points): T1 transformation and
            // energy, residual(s) and norm, and the previous iteration's update (quasi-Newton + DIIS)
            const double now = trace_ms();
            t_norm_done = now;
            std::fprintf(stderr,
                         "ccsd_gpu gs %3d  E %.12f  |Omega| %.3e  %s  %-6s moved %.3e r_c %.3e  t %.1f ms  "
                         "[T1+E %.1f  Omega %.1f  prev update %.1f]  pool %.1f/%.1f GB%s\n",
                         it, e, nrm, exact ? "fp64 " : "mixed", trace_why, trace_moved, r_c, now, t_energy,
                         now - t_start - t_energy, t_update, pool_u, pool_r,
                         fp64_final ? "  fp64 from here" : "");
        }
        if (!std::isfinite(nrm) || !std::isfinite(e)) {
            ex.prec = user;
            throw Error(CCSD_GPU_ENAN, "non-finite energy or residual in iteration " + std::to_string(it));
        }
        if (history) {
            history[2 * (it - 1)] = e;
            history[2 * (it - 1) + 1] = nrm;
        }
        norms.push_back(nrm);
        bool econv = ethr < 0 || std::fabs(e - prev) < ethr;
        if (exact && nrm < othr && econv) {
            conv = true;
            break;
        }
        // quasi-Newton step (quasi_newton_updater_class.F90, amplitude_updater_class.F90)
        qn_update(ex, omega_v.d(), epsdiff.d(), t.d(), namp, nt1);
        t1_current = false;   // the next iteration's refresh() transforms with the new t1
        // diis%update(e = scaled preconditioned residual, x = updated amplitudes)
        if (reset_diis) {
            order.clear();
            reset_diis = false;
        }
        int slot;
        if ((int)order.size() < dim) {
            slot = (int)order.size();
            order.push_back(slot);
        } else {
            slot = order.front();
            order.erase(order.begin());
            order.push_back(slot);
        }
        CU_CHECK(cudaMemcpyAsync(errs[slot].d(), omega_v.d(), sizeof(double) * namp, cudaMemcpyDeviceToDevice, s));
        CU_CHECK(cudaMemcpyAsync(pars[slot].d(), t.d(), sizeof(double) * namp, cudaMemcpyDeviceToDevice, s));
        std::vector<const double *> eptr(dim, nullptr);
        for (int k = 0; k < dim; k++) eptr[k] = errs[k].d();
        multi_dot(ex, omega_v.d(), eptr.data(), std::max<int>((int)order.size(), 1), namp, dots.d());
        DiisOrder ord{};
        ord.n = (int)order.size();
        for (int k = 0; k < ord.n; k++) ord.slot[k] = order[k];
        diis_solve(ex, Gs.d(), 16, dots.d(), slot, ord, wts.d(), stat.as<int>());
        std::vector<const double *> recs(ord.n);
        for (int k = 0; k < ord.n; k++) recs[k] = pars[order[k]].d();
        extrapolate(ex, recs.data(), wts.d(), ord.n, namp, t.d());
        int st = 0;
        CU_CHECK(cudaMemcpyAsync(&st, stat.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, s));
        CU_CHECK(cudaStreamSynchronize(s));
        if (st) {
            ex.prec = user;
            throw Error(CCSD_GPU_ESINGULAR, "could not solve DIIS matrix equation");
        }
        prev = e;
        if (trace) t_update = trace_ms() - t_norm_done;
    }
    ex.prec = user;
    refresh();
    if (trace) {
        CU_CHECK(cudaStreamSynchronize(s));
        std::fprintf(stderr, "ccsd_gpu gs done t %.1f ms\n", trace_ms());
    }
    if (energy_out) *energy_out = e;
    if (iters) *iters = it;
    return conv ? CCSD_GPU_OK : CCSD_GPU_ENOCONV;
}

// Sum of 2mnk over eT's BLAS call sites of construct_omega (DSFRK: n(n+1)k).
double Context::omega_flops() const {
    const double o = (double)no, v = (double)nv, J = (double)nJ, ov = o * v;
    const double nop = o * (o + 1) / 2, nom = o * (o - 1) / 2, nvp = v * (v + 1) / 2, nvm = v * (v - 1) / 2;
    double f = 0;
    f += 2 * J * ov * ov + 2 * v * o * J * v;                  // omega_doubles_a1
    f += 2 * ov * o * o * J + 2 * v * o * o * o * v;            // b1 (ovoo get + dgemm)
    f += 2 * ov * ov;                                           // c1
    f += 2 * ov * ov * J + 2 * v * v * v * o * o * 2 + 2 * o * o * o * v * v * 2;   // e2
    f += 2 * ov * ov * J * 2 + 2 * o * o * o * o * J + 2 * o * o * o * o * v * v * 2;   // b2
    f += 2 * v * v * o * o * J + 2 * ov * ov * J * 2 + 8 * ov * ov * ov;   // c2/d2
    f += v * v * (v * v + 1) * J + 2 * nop * nvp * nvp + 2 * nom * nvm * nvm;   // a2 (single batch)
    return f;
}

}  // namespace ccsd
