// MO Cholesky vectors from the three-index AO integrals of the Cholesky basis
// (ccsd_gpu_set_cholesky_ao), restating construct_cholesky_mo_vectors
// (src/solvers/cholesky/eri_cd_class.F90:3132-3472):
//   L_Jpq = sum_wx C_wp C_xq sum_K (wx|K) [Q^{-T}]_KJ,   S_KL = (K|L) = Q Q^T.
// eT forms (wx|K) shell block by shell block from Libint and transforms in batches; here the
// integrals arrive from the host and everything else is dense device linear algebra: S is factored
// by cuSOLVER potrf, W Q^{-T} is one triangular solve, and the two transformation products go
// through contract().
#include <cusolverDn.h>

#include "ccsd.cuh"
#include "tensor_ops.cuh"

using ccsd::Context;
using ccsd::DBuf;
using ccsd::Error;

namespace {

void solver_check(cusolverStatus_t st, const char *what) {
    if (st != CUSOLVER_STATUS_SUCCESS)
        throw Error(CCSD_GPU_ECUDA, std::string(what) + ": cusolver status " + std::to_string((int)st));
}

}  // namespace

extern "C" int ccsd_gpu_set_cholesky_ao(void *ctx, int64_t n_ao, const double *W_ao, const double *S,
                                        const double *C) {
    if (!ctx) return CCSD_GPU_EINVAL;
    Context &c = *static_cast<Context *>(ctx);
    try {
        CU_CHECK(cudaSetDevice(c.device));
        REQUIRE(n_ao > 0 && W_ao && S && C, CCSD_GPU_EINVAL, "bad AO Cholesky arguments");
        REQUIRE(n_ao >= c.nmo, CCSD_GPU_EINVAL, "n_ao smaller than the number of MOs");
        cudaStream_t s = c.ex.stream;
        const int64_t J = c.nJ, nmo = c.nmo, no = c.no, nv = c.nv, n2 = n_ao * n_ao;
        DBuf dW = ccsd::dalloc(n2 * J, s), dS = ccsd::dalloc(J * J, s), dC = ccsd::dalloc(n_ao * nmo, s);
        CU_CHECK(cudaMemcpyAsync(dW.d(), W_ao, sizeof(double) * n2 * J, cudaMemcpyHostToDevice, s));
        CU_CHECK(cudaMemcpyAsync(dS.d(), S, sizeof(double) * J * J, cudaMemcpyHostToDevice, s));
        CU_CHECK(cudaMemcpyAsync(dC.d(), C, sizeof(double) * n_ao * nmo, cudaMemcpyHostToDevice, s));
        // S = Q Q^T (lower)
        {
            cusolverDnHandle_t hs = nullptr;
            cusolverDnParams_t ps = nullptr;
            solver_check(cusolverDnCreate(&hs), "cusolverDnCreate");
            struct Guard {
                cusolverDnHandle_t h;
                cusolverDnParams_t p;
                ~Guard() {
                    if (p) cusolverDnDestroyParams(p);
                    if (h) cusolverDnDestroy(h);
                }
            } guard{hs, nullptr};
            solver_check(cusolverDnSetStream(hs, s), "cusolverDnSetStream");
            solver_check(cusolverDnCreateParams(&ps), "cusolverDnCreateParams");
            guard.p = ps;
            size_t db = 0, hb = 0;
            solver_check(cusolverDnXpotrf_bufferSize(hs, ps, CUBLAS_FILL_MODE_LOWER, J, CUDA_R_64F, dS.d(), J,
                                                     CUDA_R_64F, &db, &hb),
                         "potrf_bufferSize");
            DBuf dwork(std::max<size_t>(db, 8), s), info(sizeof(int), s);
            std::vector<char> hwork(std::max<size_t>(hb, 8));
            solver_check(cusolverDnXpotrf(hs, ps, CUBLAS_FILL_MODE_LOWER, J, CUDA_R_64F, dS.d(), J, CUDA_R_64F,
                                          dwork.as<void>(), db, hwork.data(), hb, info.as<int>()),
                         "potrf");
            int inf = 0;
            CU_CHECK(cudaMemcpyAsync(&inf, info.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, s));
            CU_CHECK(cudaStreamSynchronize(s));
            REQUIRE(inf == 0, CCSD_GPU_ESINGULAR,
                    "the Cholesky basis overlap (K|L) is not positive definite (potrf info " + std::to_string(inf) + ")");
        }
        // L_AO = W Q^{-T}: rows (w, x), columns J
        const double one = 1.0;
        BLAS_CHECK(cublasDtrsm_64(c.blas, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, CUBLAS_DIAG_NON_UNIT,
                                  n2, J, &one, dS.d(), J, dW.d(), n2));
        // L[J, p, q] = sum_wx C_wp C_xq L_AO[w, x, J]
        const ccsd::Prec keep = c.ex.prec;
        c.ex.prec = ccsd::Prec::FP64;
        DBuf T1 = ccsd::dalloc(nmo * n_ao * J, s), L = ccsd::dalloc(J * nmo * nmo, s);
        ccsd::contract(c.ex, "wxJ,wp->pxJ", 1.0, ccsd::tv(dW.d(), {n_ao, n_ao, J}), ccsd::tv(dC.d(), {n_ao, nmo}), 0.0,
                       ccsd::tv(T1.d(), {nmo, n_ao, J}));
        ccsd::contract(c.ex, "pxJ,xq->Jpq", 1.0, ccsd::tv(T1.d(), {nmo, n_ao, J}), ccsd::tv(dC.d(), {n_ao, nmo}), 0.0,
                       ccsd::tv(L.d(), {J, nmo, nmo}));
        c.ex.prec = keep;
        // the context's o/v blocks, (J, len_p, len_q) each
        auto blk = [&](DBuf &dst, int64_t p0, int64_t np, int64_t q0, int64_t nq) {
            CU_CHECK(cudaMemcpy2DAsync(dst.d(), sizeof(double) * J * np, L.d() + J * (p0 + nmo * q0),
                                       sizeof(double) * J * nmo, sizeof(double) * J * np, nq, cudaMemcpyDeviceToDevice,
                                       s));
        };
        blk(c.L_oo, 0, no, 0, no);
        blk(c.L_ov, 0, no, no, nv);
        blk(c.L_vo, no, nv, 0, no);
        blk(c.L_vv, no, nv, no, nv);
        CU_CHECK(cudaStreamSynchronize(s));
        c.have_L = true;
        c.have_gov = false;
        c.l_version++;
        if (c.have_h) c.refresh();
        c.err.clear();
        return CCSD_GPU_OK;
    } catch (const Error &e) {
        c.err = e.what();
        return e.code;
    } catch (const std::exception &e) {
        c.err = e.what();
        return CCSD_GPU_ECUDA;
    }
}
