// The CCSD residual Omega(t) recorded on a Graph, and the Jacobian transformations derived from
// it: rho = A c = (dOmega/dt) D c (forward mode) and sigma = b^T A = D (dOmega/dt)^T b (reverse
// mode), D = 2 on the packed doubles diagonal (jacobian_ccsd.F90:74-176).  Every term restates
// the routine of the eT file cited beside it.
#include <cstdio>
#include <cstdlib>
#include <memory>

#include "ccsd.cuh"
#include "ccsd_kernels.cuh"
#include "graph.cuh"
#include "mixed_gemm.cuh"
#include "tensor_ops.cuh"

namespace ccsd {

namespace {

#define GRID_STRIDE(i, total) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (total); i += (int64_t)gridDim.x * blockDim.x)

inline int grid_for(int64_t total, int block) {
    int64_t g = (total + block - 1) / block;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 64));
}

// [t1 | t2] columns <-> separate (nt1 x n) and (nt2 x n) arrays, with the doubles diagonal scaled
__global__ void split_amp_kernel(const double *__restrict__ x, int64_t nt1, int64_t nov, int64_t nvec, double diag,
                                 double *__restrict__ x1, double *__restrict__ x2) {
    const int64_t nt2 = nov * (nov + 1) / 2, namp = nt1 + nt2;
    GRID_STRIDE(idx, namp * nvec) {
        int64_t n = idx / namp, k = idx - n * namp;
        double v = x[idx];
        if (k < nt1) x1[n * nt1 + k] = v;
        else {
            int64_t p = k - nt1;
            int64_t M = (int64_t)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
            while (M * (M + 1) / 2 > p) M--;
            while ((M + 1) * (M + 2) / 2 <= p) M++;
            if (p - M * (M + 1) / 2 == M) v *= diag;
            x2[n * nt2 + p] = v;
        }
    }
}

__global__ void join_amp_kernel(const double *__restrict__ x1, const double *__restrict__ x2, int64_t nt1, int64_t nov,
                                int64_t nvec, double diag, double *__restrict__ x) {
    const int64_t nt2 = nov * (nov + 1) / 2, namp = nt1 + nt2;
    GRID_STRIDE(idx, namp * nvec) {
        int64_t n = idx / namp, k = idx - n * namp;
        if (k < nt1) x[idx] = x1[n * nt1 + k];
        else {
            int64_t p = k - nt1;
            int64_t M = (int64_t)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
            while (M * (M + 1) / 2 > p) M--;
            while ((M + 1) * (M + 2) / 2 <= p) M++;
            double v = x2[n * nt2 + p];
            if (p - M * (M + 1) / 2 == M) v *= diag;
            x[idx] = v;
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Omega on the graph
// ---------------------------------------------------------------------------
OmegaNodes Context::record_omega(Graph &g, bool const_ovov, bool const_t1) {
    OmegaNodes n{};
    g.nov = nov;
    const std::vector<int64_t> V4 = {nv, no, nv, no};
    n.t1 = g.input("t1", {nv, no}, t.d());
    n.t2 = g.input("t2", {nt2}, t.d() + nt1);
    n.L_oo = g.input("L_oo", {nJ, no, no}, L_oo.d());
    n.L_ov = g.input("L_ov", {nJ, no, nv}, L_ov.d());
    n.L_vo = g.input("L_vo", {nJ, nv, no}, L_vo.d());
    n.L_vv = g.input("L_vv", {nJ, nv, nv}, L_vv.d());
    n.h_oo = g.input("h_oo", {no, no}, hb_oo.d());
    n.h_ov = g.input("h_ov", {no, nv}, hb_ov.d());
    n.h_vo = g.input("h_vo", {nv, no}, hb_vo.d());
    n.h_vv = g.input("h_vv", {nv, nv}, hb_vv.d());
    const int t1 = n.t1;

    int Lt_ov, Lt_oo, Lt_vo, Lt_vv, F_oo, F_ov, F_vo, F_vv;
    if (const_t1) {
        // the context transformed the blocks and built the Fock matrix at this t1 (refresh())
        Lt_oo = g.input("Lt_oo", {nJ, no, no}, this->Lt_oo.d());
        Lt_ov = g.input("Lt_ov", {nJ, no, nv}, this->Lt_ov.d());
        Lt_vo = g.input("Lt_vo", {nJ, nv, no}, this->Lt_vo.d());
        Lt_vv = g.input("Lt_vv", {nJ, nv, nv}, this->Lt_vv.d());
        F_oo = g.input("F_oo", {no, no}, fb_oo.d());
        F_ov = g.input("F_ov", {no, nv}, fb_ov.d());
        F_vo = g.input("F_vo", {nv, no}, fb_vo.d());
        F_vv = g.input("F_vv", {nv, nv}, fb_vv.d());
        n.Lt_vv = Lt_vv;
    } else {
        // construct_t1_cholesky (src/wavefunctions/ccs/t1_ccs.F90:208-499); the ov block is unchanged
        auto t1_timer = std::make_unique<TermTimer>(ex, "T1 transform cholesky");
        Lt_ov = g.alias(n.L_ov);
        Lt_oo = g.zeros("Lt_oo", {nJ, no, no});
        g.permute(Lt_oo, "Jij->Jij", 1.0, n.L_oo);
        g.contract(Lt_oo, "Jia,aj->Jij", 1.0, n.L_ov, t1, true);
        Lt_vo = g.zeros("Lt_vo", {nJ, nv, no});
        g.permute(Lt_vo, "Jai->Jai", 1.0, n.L_vo);
        g.contract(Lt_vo, "Jab,bi->Jai", 1.0, n.L_vv, t1, true);
        g.contract(Lt_vo, "aj,Jji->Jai", -1.0, t1, Lt_oo, true);
        Lt_vv = g.zeros("Lt_vv", {nJ, nv, nv});
        g.permute(Lt_vv, "Jab->Jab", 1.0, n.L_vv);
        g.contract(Lt_vv, "aj,Jjb->Jab", -1.0, t1, n.L_ov, true);
        n.Lt_vv = Lt_vv;
        t1_timer.reset();

        // T1 Fock matrix in blocks (fock_ccs.F90:242-1107): h~ = (1 - t1) h (1 + t1) then
        // F_pq = h~_pq + 2 sum_J L~_pq X_J - sum_Jk L~_pk L~_kq, X_J = sum_k L~_kk
        auto fock_timer = std::make_unique<TermTimer>(ex, "Fock matrix construction (T1 basis)");
        F_oo = g.zeros("F_oo", {no, no});
        F_ov = g.zeros("F_ov", {no, nv});
        F_vo = g.zeros("F_vo", {nv, no});
        F_vv = g.zeros("F_vv", {nv, nv});
        g.permute(F_oo, "ij->ij", 1.0, n.h_oo);
        g.contract(F_oo, "ia,aj->ij", 1.0, n.h_ov, t1, true);          // h~_oo = h_oo + h_ov t1
        g.permute(F_ov, "ia->ia", 1.0, n.h_ov);                          // h~_ov = h_ov
        g.permute(F_vv, "ab->ab", 1.0, n.h_vv);
        g.contract(F_vv, "ai,ib->ab", -1.0, t1, n.h_ov, true);          // h~_vv = h_vv - t1 h_ov
        const int Woo = g.zeros("W_oo", {no, no});
        g.permute(Woo, "ij->ij", 1.0, n.h_oo);
        g.contract(Woo, "ia,aj->ij", 1.0, n.h_ov, t1, true);
        g.permute(F_vo, "ai->ai", 1.0, n.h_vo);
        g.contract(F_vo, "ab,bi->ai", 1.0, n.h_vv, t1, true);
        g.contract(F_vo, "aj,ji->ai", -1.0, t1, Woo, true);             // h~_vo = h_vo + h_vv t1 - t1 W_oo
        const int X = g.zeros("X_J", {nJ});
        g.trace(X, Lt_oo);
        g.contract(F_oo, "Jpq,J->pq", 2.0, Lt_oo, X, true);
        g.contract(F_ov, "Jpq,J->pq", 2.0, Lt_ov, X, true);
        g.contract(F_vo, "Jpq,J->pq", 2.0, Lt_vo, X, true);
        g.contract(F_vv, "Jpq,J->pq", 2.0, Lt_vv, X, true);
        g.contract(F_oo, "Jpk,Jkq->pq", -1.0, Lt_oo, Lt_oo, true);
        g.contract(F_ov, "Jpk,Jkq->pq", -1.0, Lt_oo, Lt_ov, true);
        g.contract(F_vo, "Jpk,Jkq->pq", -1.0, Lt_vo, Lt_oo, true);
        g.contract(F_vv, "Jpk,Jkq->pq", -1.0, Lt_vo, Lt_ov, true);
        fock_timer.reset();
    }

    // construct_omega_ccsd (src/wavefunctions/ccsd/omega_ccsd.F90:39-110)
    const int om1 = g.zeros("omega1", {nv, no});
    g.permute(om1, "ai->ai", 1.0, F_vo);                            // omega_ccs_a1 (omega_ccs.F90:62)
    const int tf = g.zeros("t_aibj", V4);
    const int u = g.zeros("u_aibj", V4);                             // construct_u_aibj (omega_ccsd.F90:881)
    {
        TermTimer tt(ex, "Construct u_aibj");
        g.squareup(tf, n.t2);                                        // squareup (reordering.F90:4174)
        g.permute(u, "aibj->aibj", 2.0, tf);
        g.permute(u, "ajbi->aibj", -1.0, tf);
    }
    {
        // omega_doubles_a1 (src/wavefunctions/doubles/omega_doubles.F90:36-138)
        TermTimer tt(ex, "omega doubles a1");
        const int XJ = g.zeros("X_Jbi", {nJ, nv, no});
        g.contract(XJ, "Jcj,cjbi->Jbi", 1.0, n.L_vo, u);
        g.contract(om1, "Jab,Jbi->ai", 1.0, Lt_vv, XJ);
    }
    {
        // omega_doubles_b1 (:141-204)
        TermTimer tt(ex, "omega doubles b1");
        const int gkbji = g.zeros("g_kbji", {no, nv, no, no});
        g.contract(gkbji, "Jkb,Jji->kbji", 1.0, Lt_ov, Lt_oo);
        g.contract(om1, "ajbk,kbji->ai", -1.0, u, gkbji);
    }
    {
        // omega_doubles_c1 (:207-258)
        TermTimer tt(ex, "omega doubles c1");
        g.contract(om1, "aibj,jb->ai", 1.0, u, F_ov, true);
    }

    // g_ldkc, shared below (FP64 cache unless the adjoint into L_ov is wanted)
    int G4;
    if (const_ovov) {
        G4 = g.input("g_ovov", {no, nv, no, nv}, g_ovov_const());
    } else {
        G4 = g.zeros("g_ovov", {no, nv, no, nv});
        g.contract(G4, "Jia,Jjb->iajb", 1.0, Lt_ov, Lt_ov);
    }
    // omega_ccsd_e2 (omega_ccsd.F90:712-878); Fock parts in FP64
    const int om = g.zeros("omega_aibj", V4);
    {
        TermTimer tt(ex, "omega ccsd e2");
        const int Xbc = g.zeros("X_bc", {nv, nv}), Ykj = g.zeros("Y_kj", {no, no});
        g.contract(Xbc, "bkdl,ldkc->bc", -1.0, u, G4);
        g.contract(Ykj, "kdlc,djcl->kj", 1.0, G4, u);
        // the Fock blocks join X and Y, so each side is one FP64 product with t (the Fock parts are
        // first-order terms)
        g.permute(Xbc, "bc->bc", 1.0, F_vv);
        g.permute(Ykj, "kj->kj", 1.0, F_oo);
        g.contract(om, "bc,cjai->bjai", 1.0, Xbc, tf, true);
        g.contract(om, "aibk,kj->aibj", -1.0, tf, Ykj, true);
    }
    // om collects the terms that eT symmetrises (symmetric_sum, reordering.F90:416): the doubles
    // residual is pack(om + om^T) with the diagonal halved, formed in one pass at the end.  Terms
    // that are symmetric already enter with weight 1/2.
    // omega_ccsd_b2 (omega_ccsd.F90:483-583); g_aibj in FP64
    {
        TermTimer tt(ex, "omega ccsd b2");
        g.contract(om, "Jai,Jbj->aibj", 0.5, Lt_vo, Lt_vo, true);
        const int X4 = g.zeros("X_klij", {no, no, no, no});
        g.contract(X4, "Jki,Jlj->klij", 1.0, Lt_oo, Lt_oo);
        g.contract(X4, "kcld,cidj->klij", 1.0, G4, tf);
        g.contract(om, "akbl,klij->aibj", 0.5, tf, X4);
    }
    // omega_ccsd_c2_d2 (omega_ccsd.F90:586-709) in contraction form
    {
        TermTimer tt(ex, "omega ccsd c2 and d2");
        const int C = g.zeros("C_term", V4), D = g.zeros("D_term", V4);
        g.contract(C, "Jac,Jkj->ckaj", 1.0, Lt_vv, Lt_oo);
        g.permute(D, "ckaj->ckaj", -1.0, C);
        g.contract(D, "Jai,Jkc->ckai", 2.0, Lt_vo, Lt_ov);
        g.contract(C, "kcld,djak->claj", -0.5, G4, tf);
        // the two g_ovov terms of D share u: one contraction with H_lckd = g_lckd - 1/2 g_kcld
        int H;
        if (const_ovov) {
            H = g.input("H_lckd", {no, nv, no, nv}, h_ovov_const());
        } else {
            H = g.zeros("H_lckd", {no, nv, no, nv});
            g.permute(H, "lckd->lckd", 1.0, G4);
            g.permute(H, "kcld->lckd", -0.5, G4);
        }
        g.contract(D, "lckd,dkaj->claj", 1.0, H, u);
        const int x = g.zeros("x_c2", V4);
        g.contract(x, "akci,ckbj->aibj", -1.5, tf, C);
        g.contract(om, "aick,ckbj->aibj", 0.5, u, D);
        g.permute(om, "aibj->aibj", 1.0 / 3.0, x);
        g.permute(om, "ajbi->aibj", 2.0 / 3.0, x);
    }
    const int om2 = g.zeros("omega2", {nt2});
    g.pack_sym(om2, om);                     // symmetric_sum + scale_diagonal(1/2) + packin
    // omega_ccsd_a2 (omega_ccsd.F90:113-480) as a custom op
    record_ladder(g, om2, Lt_vv, n.t2, t1, n.L_vv, tf);
    n.om1 = om1;
    n.om2 = om2;
    return n;
}

// Y[k,i,b,j] = sum_cd g_kcbd t_cidj with g_kcbd = sum_J L_kc L~_bd (batched over b; in mixed
// precision the residual and the derivatives take Y from the resident ovvv planes instead)
void Context::ladder_y(const double *Lvv, const double *tfull, double *Y) {
    cudaStream_t s = ex.stream;
    const int64_t nb = std::max<int64_t>(1, std::min<int64_t>(nv, (int64_t)(2.0e9 / (8.0 * no * nv * nv))));
    DBuf gblk = dalloc(no * nv * nb * nv, s);
    for (int64_t b0 = 0; b0 < nv; b0 += nb) {
        const int64_t b1 = std::min(nv, b0 + nb), len = b1 - b0;
        TV Lb = tv(Lvv + nJ * b0, {nJ, len, nv});
        Lb.s[1] = nJ;
        Lb.s[2] = nJ * nv;
        TV gb = tv(gblk.d(), {no, nv, len, nv});
        contract(ex, "Jkc,Jbd->kcbd", 1.0, tv(L_ov.d(), {nJ, no, nv}), Lb, 0.0, gb);
        TV Yb = tv(Y + no * no * b0, {no, no, len, no});
        Yb.s[1] = no;
        Yb.s[2] = no * no;
        Yb.s[3] = no * no * nv;
        contract(ex, "kcbd,cidj->kibj", 1.0, gb, tv(tfull, {nv, no, nv, no}), 0.0, Yb);
    }
}

void Context::record_ladder(Graph &g, int om2, int Lvv, int t2, int t1, int L_vv_in, int tf) {
    auto Ycache = std::make_shared<DBuf>();
    auto LTcache = std::make_shared<DBuf>();
    auto getY = [this, &g, Lvv, t1, tf, Ycache]() -> const double * {
        if (!*Ycache) {
            *Ycache = dalloc(no * no * nv * no, ex.stream);
            ladder_y_t1(g.value(t1), g.value(Lvv), g.value(tf), Ycache->d());
        }
        return Ycache->d();
    };
    auto getLT = [this, &g, Lvv, LTcache]() -> const double * {
        if (!*LTcache) {
            *LTcache = dalloc(nJ * nv * nv, ex.stream);
            TV src = tv(g.value(Lvv), {nJ, nv, nv});
            TV dst = tv(LTcache->d(), {nJ, nv, nv});
            dst.s[1] = nJ * nv;
            dst.s[2] = nJ;
            permute_add(ex, 1.0, src, 0.0, dst);
        }
        return LTcache->d();
    };
    CustomOp op;
    op.forward = [this, &g, om2, Lvv, t2, t1, tf]() {
        TermTimer tt(ex, "omega ccsd a2");
        if (ex.prec == Prec::MIXED)
            ladder_residual_mixed(g.value(t1), g.value(tf), g.value(t2), g.node(om2).v);
        else if (f64_resident())
            ladder_residual_f64(g.value(t1), g.value(tf), g.value(t2), g.node(om2).v);
        else
            ladder(g.value(Lvv), g.value(t2), g.node(om2).v);
    };
    op.tangent = [this, &g, om2, Lvv, t2, t1, getY](int nvec) {
        REQUIRE(!g.node(Lvv).active || g.node(t1).active, CCSD_GPU_EINVAL,
                "ladder tangent: L_vv directions are not supported");
        double *out = g.tangent(om2, nvec);
        if (g.node(t2).active) {
            const double *c2 = g.tangent(t2, nvec);
            ladder(g.value(Lvv), c2, out, nvec);
        }
        if (g.node(t1).active) {
            // d L~_ac = -sum_k c_ak L_kc: term -P(sum_k c_ak Y_kibj + (ai <-> bj))
            const double *Y = getY();
            const double *c1 = g.tangent(t1, nvec);
            DBuf A = dalloc(nov * nov, ex.stream);
            for (int n = 0; n < nvec; n++) {
                contract(ex, "ak,kibj->aibj", -1.0, tv(c1 + n * nt1, {nv, no}), tv(Y, {no, no, nv, no}), 0.0,
                         tv(A.d(), {nv, no, nv, no}));
                pack_sym_add(ex, A.d(), out + n * nt2, nov);   // pack(A + A^T), diagonal halved
            }
        }
    };
    op.adjoint = [this, &g, om2, Lvv, t2, t1, tf, L_vv_in, getY, getLT](int nvec) {
        // adjoint into the Cholesky vectors requested: dense route through L~_vv (its adjoint also
        // reaches t1 through the recorded T1 transformation); otherwise the rank-n_o route via Y
        const bool dense = g.node(L_vv_in).active;
        const double *pbar = g.adjoint(om2, nvec);
        if (g.node(t2).active) {
            // the transpose of the packed ladder is the same ladder with L~_vv transposed
            const double *LT = getLT();
            double *t2bar = g.adjoint(t2, nvec);
            ladder(LT, pbar, t2bar, nvec);
        }
        if (g.node(t1).active || dense) {
            DBuf B = dalloc(nov * nov, ex.stream);
            for (int n = 0; n < nvec; n++) {
                squareup(ex, pbar + n * nt2, B.d(), nov);
                if (g.node(t1).active && !dense) {
                    // t1bar_ak -= sum_ibj S(pbar)_aibj Y_kibj
                    contract(ex, "aibj,kibj->ak", -1.0, tv(B.d(), {nv, no, nv, no}), tv(getY(), {no, no, nv, no}),
                             1.0, tv(g.adjoint(t1, nvec) + n * nt1, {nv, no}));
                }
                if (dense) {
                    // Lbar_J,ac += sum_bd L_J,bd Z_acbd, Z_acbd = sum_ij S(pbar)_aibj t_cidj
                    REQUIRE((double)nv * nv * nv * nv * 8.0 < 24e9, CCSD_GPU_EINVAL,
                            "ladder adjoint into L_vv needs v^4 doubles of scratch; system too large");
                    DBuf Z = dalloc(nv * nv * nv * nv, ex.stream);
                    contract(ex, "aibj,cidj->acbd", 1.0, tv(B.d(), {nv, no, nv, no}), tv(g.value(tf), {nv, no, nv, no}),
                             0.0, tv(Z.d(), {nv, nv, nv, nv}));
                    contract(ex, "Jbd,acbd->Jac", 1.0, tv(g.value(Lvv), {nJ, nv, nv}), tv(Z.d(), {nv, nv, nv, nv}), 1.0,
                             tv(g.adjoint(Lvv, nvec) + n * nJ * nv * nv, {nJ, nv, nv}));
                }
            }
        }
    };
    g.custom(std::move(op), om2, {Lvv, t2, t1, tf});
}

void Context::omega_eager(double *om_out) {
    Graph g(ex);
    OmegaNodes n = record_omega(g, true, t1_current);
    CU_CHECK(cudaMemcpyAsync(om_out, g.value(n.om1), sizeof(double) * nt1, cudaMemcpyDeviceToDevice, ex.stream));
    CU_CHECK(cudaMemcpyAsync(om_out + nt1, g.value(n.om2), sizeof(double) * nt2, cudaMemcpyDeviceToDevice, ex.stream));
}

void Context::prepare_residual_caches() {
    g_ovov_const();
    if (ex.prec == Prec::MIXED) {
        if (ladder_pairs_resident()) ladder_pairs(L_vv.d(), true);
        if (ovvv_resident()) ovvv_pairs();
    } else if (f64_resident()) {
        f64_integrals();
    }
}

// Records the residual on ex.stream into G.  A capture that fails (a call that cannot be captured)
// leaves G empty and turns graphs off for this context; the caller then evaluates eagerly.
void Context::capture_residual(ResidualGraph &G, double *om_out) {
    G.reset();
    graphs_captured = true;
    const double flops0 = ex.flops;
    const int64_t launches0 = ex.launches;
    cudaGraph_t graph = nullptr;
    std::string why;
    CU_CHECK(cudaStreamBeginCapture(ex.stream, cudaStreamCaptureModeThreadLocal));
    try {
        omega_eager(om_out);
    } catch (const std::exception &e) {
        why = e.what();
    }
    cudaError_t rc = cudaStreamEndCapture(ex.stream, &graph);
    if (why.empty() && rc == cudaSuccess && graph) {
        rc = cudaGraphInstantiate(&G.exec, graph, 0);
        if (rc != cudaSuccess) G.exec = nullptr;
    }
    if (graph) cudaGraphDestroy(graph);
    if (!G.exec) {
        if (why.empty()) why = cudaGetErrorString(rc);
        cudaGetLastError();
        use_graphs = false;
        if (std::getenv("CCSD_GPU_TRACE"))
            std::fprintf(stderr, "ccsd_gpu residual graph capture failed (%s); evaluating eagerly\n", why.c_str());
    }
    G.flops = ex.flops - flops0;
    G.launches = ex.launches - launches0;
    ex.flops = flops0;
    ex.launches = launches0;
    G.l_version = l_version;
    G.cache_epoch = cache_epoch;
    G.planes = ex.planes;
    G.k_chunk = ex.k_chunk;
}

void Context::omega(double *om_out) {
    REQUIRE(have_t, CCSD_GPU_ESTATE, "amplitudes not set");
    if (!t1_current) refresh();   // the residual reads the context's T1-transformed blocks
    TermTimer tt(ex, "Construct CCSD Omega");
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CU_CHECK(cudaStreamIsCapturing(ex.stream, &cap));
    const bool graphs = use_graphs && !(ex.prof && ex.prof->on) && cap == cudaStreamCaptureStatusNone;
    if (!graphs) {
        omega_eager(om_out);
    } else {
        prepare_residual_caches();
        ResidualGraph &G = rgraph[ex.prec == Prec::MIXED ? 1 : 0];
        if (!G.warm) {
            omega_eager(om_out);
            G.warm = true;
        } else {
            // the graph writes a buffer of its own, so callers may pass any output
            if (!om_stage) om_stage = dalloc(namp, ex.stream);
            const bool match = G.exec && G.l_version == l_version && G.cache_epoch == cache_epoch &&
                               G.planes == ex.planes && G.k_chunk == ex.k_chunk;
            if (!match) capture_residual(G, om_stage.d());
            if (G.exec) {
                CU_CHECK(cudaGraphLaunch(G.exec, ex.stream));
                CU_CHECK(cudaMemcpyAsync(om_out, om_stage.d(), sizeof(double) * namp, cudaMemcpyDeviceToDevice,
                                         ex.stream));
                ex.flops += G.flops;
                ex.launches += G.launches;
                graph_replays++;
            } else {
                omega_eager(om_out);
            }
        }
    }
    check_gemm();
}

void Context::check_gemm() {
    const int code = gemm_error(ex, true);
    REQUIRE(code == 0, CCSD_GPU_ETIMEOUT,
            "tensor-core GEMM barrier wait timed out (code " + std::to_string(code) + ")");
}

// prepare_for_jacobian (jacobian_ccsd.F90:46-71) / prepare_for_jacobian_transpose
// (jacobian_transpose_ccsd.F90:44-126): eT computes and stores the t-dependent intermediates of its
// hand-written terms once per Davidson run; here the whole residual is recorded once at the current
// amplitudes, so every later transformation runs only its derivative pass over the stored values.
void Context::prepare_jacobian() {
    REQUIRE(have_t, CCSD_GPU_ESTATE, "amplitudes not set");
    drop_jacobian();
    auto p = std::make_unique<PreparedJacobian>();
    p->g = std::make_unique<Graph>(ex);
    p->n = record_omega(*p->g);
    p->prec = ex.prec;
    p->planes = ex.planes;
    p->k_chunk = ex.k_chunk;
    p->l_version = l_version;
    p->id = ++prep_counter;
    CU_CHECK(cudaStreamSynchronize(ex.stream));
    check_gemm();
    prep = std::move(p);
}

void Context::drop_jacobian() {
    if (!prep) return;
    prep.reset();
    if (mbuf_kind == 2) mbuf_reuse = -1;
}

Graph &Context::transform_graph(std::unique_ptr<Graph> &local, OmegaNodes &n) {
    if (prep && prep->prec == ex.prec && prep->planes == ex.planes && prep->k_chunk == ex.k_chunk &&
        prep->l_version == l_version) {
        n = prep->n;
        pairs_reuse_id = prep->id;
        return *prep->g;
    }
    local = std::make_unique<Graph>(ex);
    n = record_omega(*local);
    return *local;
}

namespace {
// a prepared transformation's ladder integrals stay reusable only while it runs
struct ReuseScope {
    int64_t &id;
    ~ReuseScope() { id = -1; }
};
}  // namespace

// rho_k = A c_k for n_vec device columns [t1 | packed t2]
void Context::jacobian(int64_t nvec, const double *c, double *rho) {
    REQUIRE(have_t, CCSD_GPU_ESTATE, "amplitudes not set");
    TermTimer tt(ex, "Jacobian CCSD transformation");
    ReuseScope scope{pairs_reuse_id};
    std::unique_ptr<Graph> local;
    OmegaNodes n;
    Graph &g = transform_graph(local, n);
    DBuf s1 = dalloc(nt1 * nvec, ex.stream), s2 = dalloc(nt2 * nvec, ex.stream);
    split_amp_kernel<<<grid_for(namp * nvec, 256), 256, 0, ex.stream>>>(c, nt1, nov, nvec, 2.0, s1.d(), s2.d());
    ex.launches++;
    DBuf r1 = dalloc(nt1 * nvec, ex.stream), r2 = dalloc(nt2 * nvec, ex.stream);
    g.jvp({n.t1, n.t2}, {s1.d(), s2.d()}, (int)nvec, {n.om1, n.om2}, {r1.d(), r2.d()});
    join_amp_kernel<<<grid_for(namp * nvec, 256), 256, 0, ex.stream>>>(r1.d(), r2.d(), nt1, nov, nvec, 1.0, rho);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
    g.clear_derivatives();
    CU_CHECK(cudaStreamSynchronize(ex.stream));
    check_gemm();
}

// sigma_k = b_k^T A = D (dOmega/dt)^T b_k
void Context::jacobian_transpose(int64_t nvec, const double *b, double *sigma) {
    REQUIRE(have_t, CCSD_GPU_ESTATE, "amplitudes not set");
    TermTimer tt(ex, "Jacobian transpose CCSD");
    ReuseScope scope{pairs_reuse_id};
    std::unique_ptr<Graph> local;
    OmegaNodes n;
    Graph &g = transform_graph(local, n);
    DBuf s1 = dalloc(nt1 * nvec, ex.stream), s2 = dalloc(nt2 * nvec, ex.stream);
    split_amp_kernel<<<grid_for(namp * nvec, 256), 256, 0, ex.stream>>>(b, nt1, nov, nvec, 1.0, s1.d(), s2.d());
    ex.launches++;
    DBuf r1 = dalloc(nt1 * nvec, ex.stream), r2 = dalloc(nt2 * nvec, ex.stream);
    g.vjp({n.om1, n.om2}, {s1.d(), s2.d()}, (int)nvec, {n.t1, n.t2}, {r1.d(), r2.d()});
    join_amp_kernel<<<grid_for(namp * nvec, 256), 256, 0, ex.stream>>>(r1.d(), r2.d(), nt1, nov, nvec, 2.0, sigma);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
    g.clear_derivatives();
    CU_CHECK(cudaStreamSynchronize(ex.stream));
    check_gemm();
}

// b^T dOmega/d(t, L, h): amplitude part without the D scaling, plus the adjoints into the MO
// Cholesky blocks (J, p, q) and the MO one-electron Hamiltonian (n_mo x n_mo, column-major)
void Context::adjoint(const double *b, double *dt, double *dL, double *dh) {
    REQUIRE(have_t, CCSD_GPU_ESTATE, "amplitudes not set");
    Graph g(ex);
    OmegaNodes n = record_omega(g, dL == nullptr);
    DBuf s1 = dalloc(nt1, ex.stream), s2 = dalloc(nt2, ex.stream);
    split_amp_kernel<<<grid_for(namp, 256), 256, 0, ex.stream>>>(b, nt1, nov, 1, 1.0, s1.d(), s2.d());
    ex.launches++;
    std::vector<int> ins = {n.t1, n.t2};
    std::vector<DBuf> outs;
    outs.push_back(dalloc(nt1, ex.stream));
    outs.push_back(dalloc(nt2, ex.stream));
    const bool wantL = dL != nullptr, wanth = dh != nullptr;
    if (wantL)
        for (int node : {n.L_oo, n.L_ov, n.L_vo, n.L_vv}) {
            ins.push_back(node);
            outs.push_back(dalloc(g.node(node).size, ex.stream));
        }
    if (wanth)
        for (int node : {n.h_oo, n.h_ov, n.h_vo, n.h_vv}) {
            ins.push_back(node);
            outs.push_back(dalloc(g.node(node).size, ex.stream));
        }
    std::vector<double *> res;
    for (auto &o : outs) res.push_back(o.d());
    g.vjp({n.om1, n.om2}, {s1.d(), s2.d()}, 1, ins, res);
    if (dt) {
        join_amp_kernel<<<grid_for(namp, 256), 256, 0, ex.stream>>>(outs[0].d(), outs[1].d(), nt1, nov, 1, 1.0, dt);
        ex.launches++;
    }
    size_t k = 2;
    auto scatter = [&](double *full, int64_t ld, int64_t p0, int64_t q0, int64_t np, int64_t nq, const double *blk,
                       int64_t inner) {
        // full[(inner) x (p0+p) x (q0+q)] <- blk[inner x p x q]
        TV src = tv(blk, {inner, np, nq});
        TV dst;
        dst.p = full + inner * (p0 + ld * q0);
        dst.nd = 3;
        dst.n[0] = inner;
        dst.n[1] = np;
        dst.n[2] = nq;
        dst.s[0] = 1;
        dst.s[1] = inner;
        dst.s[2] = inner * ld;
        permute_add(ex, 1.0, src, 0.0, dst);
    };
    if (wantL) {
        scatter(dL, nmo, 0, 0, no, no, outs[k++].d(), nJ);
        scatter(dL, nmo, 0, no, no, nv, outs[k++].d(), nJ);
        scatter(dL, nmo, no, 0, nv, no, outs[k++].d(), nJ);
        scatter(dL, nmo, no, no, nv, nv, outs[k++].d(), nJ);
    }
    if (wanth) {
        scatter(dh, nmo, 0, 0, no, no, outs[k++].d(), 1);
        scatter(dh, nmo, 0, no, no, nv, outs[k++].d(), 1);
        scatter(dh, nmo, no, 0, nv, no, outs[k++].d(), 1);
        scatter(dh, nmo, no, no, nv, nv, outs[k++].d(), 1);
    }
    CU_CHECK(cudaGetLastError());
    CU_CHECK(cudaStreamSynchronize(ex.stream));
    check_gemm();
}

}  // namespace ccsd
