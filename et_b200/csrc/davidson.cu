// Davidson solver for the lowest EOM-CCSD roots of A (right) or A^T (left), restating
// eigen_davidson_solver (src/solvers/eigen_davidson_solver_class.F90:122-229) and
// eigen_davidson_tool / davidson_tool (src/solver_tools/davidson/): trial vectors, their
// transforms and the reduced space live in HBM; new trials are transformed as one block through
// the batched Jacobian; the reduced non-symmetric eigenproblem is solved in FP64 on the device
// (cuSOLVER geev).
#include <cusolverDn.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <numeric>

#include "ccsd.cuh"
#include "ccsd_kernels.cuh"
#include "tensor_ops.cuh"

namespace ccsd {

namespace {
// A Davidson run prepares the transformations once (eT calls prepare_for_jacobian before its
// solver loop) and drops what it prepared when it ends; a preparation the caller made is kept.
struct PrepareScope {
    Context &c;
    bool own;
    explicit PrepareScope(Context &ctx) : c(ctx), own(!ctx.prep) {
        if (own) c.prepare_jacobian();
    }
    ~PrepareScope() {
        if (own) c.drop_jacobian();
    }
};
}  // namespace

namespace {

#define SOLVER_CHECK(x)                                                                        \
    do {                                                                                       \
        cusolverStatus_t st__ = (x);                                                           \
        if (st__ != CUSOLVER_STATUS_SUCCESS)                                                   \
            throw ::ccsd::Error(CCSD_GPU_ECUDA, std::string(#x) + ": cusolver status " +       \
                                std::to_string((int)st__));                                    \
    } while (0)

#define GRID_STRIDE(i, total) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (total); i += (int64_t)gridDim.x * blockDim.x)

inline int grid_for(int64_t total, int block) {
    int64_t g = (total + block - 1) / block;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 64));
}

// new trial = residual / (omega - eps) (orbital-difference preconditioner, davidson_tool)
__global__ void precondition_kernel(const double *__restrict__ r, const double *__restrict__ eps, double omega,
                                    int64_t n, double *__restrict__ out) {
    GRID_STRIDE(i, n) {
        double d = omega - eps[i];
        if (fabs(d) < 1e-8) d = d < 0 ? -1e-8 : 1e-8;
        out[i] = r[i] / d;
    }
}

__global__ void unit_vector_kernel(double *__restrict__ v, int64_t n, int64_t k) {
    GRID_STRIDE(i, n) { v[i] = (i == k) ? 1.0 : 0.0; }
}

struct Geev {
    cusolverDnHandle_t h = nullptr;
    cusolverDnParams_t p = nullptr;
    Geev(cudaStream_t s) {
        SOLVER_CHECK(cusolverDnCreate(&h));
        SOLVER_CHECK(cusolverDnSetStream(h, s));
        SOLVER_CHECK(cusolverDnCreateParams(&p));
    }
    ~Geev() {
        if (p) cusolverDnDestroyParams(p);
        if (h) cusolverDnDestroy(h);
    }
    // eigenvalues (complex) and right eigenvectors (LAPACK real packing) of the dim x dim matrix G (device)
    void solve(cudaStream_t s, double *G, int64_t dim, std::vector<std::complex<double>> &w, std::vector<double> &vr) {
        DBuf W(sizeof(double) * 2 * dim, s), VR = dalloc(dim * dim, s);
        size_t dbytes = 0, hbytes = 0;
        SOLVER_CHECK(cusolverDnXgeev_bufferSize(h, p, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, dim,
                                                CUDA_R_64F, G, dim, CUDA_C_64F, W.as<void>(), CUDA_R_64F, nullptr,
                                                dim, CUDA_R_64F, VR.as<void>(), dim, CUDA_R_64F, &dbytes, &hbytes));
        DBuf dwork(std::max<size_t>(dbytes, 8), s);
        std::vector<char> hwork(std::max<size_t>(hbytes, 8));
        DBuf info(sizeof(int), s);
        SOLVER_CHECK(cusolverDnXgeev(h, p, CUSOLVER_EIG_MODE_NOVECTOR, CUSOLVER_EIG_MODE_VECTOR, dim, CUDA_R_64F, G,
                                     dim, CUDA_C_64F, W.as<void>(), CUDA_R_64F, nullptr, dim, CUDA_R_64F,
                                     VR.as<void>(), dim, CUDA_R_64F, dwork.as<void>(), dbytes, hwork.data(), hbytes,
                                     info.as<int>()));
        int inf = 0;
        CU_CHECK(cudaMemcpyAsync(&inf, info.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, s));
        w.resize(dim);
        vr.resize(dim * dim);
        CU_CHECK(cudaMemcpyAsync(w.data(), W.as<void>(), sizeof(double) * 2 * dim, cudaMemcpyDeviceToHost, s));
        CU_CHECK(cudaMemcpyAsync(vr.data(), VR.d(), sizeof(double) * dim * dim, cudaMemcpyDeviceToHost, s));
        CU_CHECK(cudaStreamSynchronize(s));
        REQUIRE(inf == 0, CCSD_GPU_ESINGULAR, "reduced eigenproblem (geev) failed, info " + std::to_string(inf));
    }
};

}  // namespace

int Context::davidson(int nstates, int side, const ccsd_gpu_davidson_options *o, double *omega_out,
                      double *vectors_out, int32_t *iters_out, const double *start) {
    REQUIRE(have_t && have_L && have_h, CCSD_GPU_ESTATE, "inputs/amplitudes not set");
    REQUIRE(nstates > 0 && nstates <= namp, CCSD_GPU_EINVAL, "bad number of states");
    cudaStream_t s = ex.stream;
    const int maxit = o && o->max_iterations > 0 ? o->max_iterations : 100;
    const double rthr = o && o->residual_threshold > 0 ? o->residual_threshold : 1e-6;
    const double ethr = o && o->energy_threshold > 0 ? o->energy_threshold : 1e-6;
    const int64_t maxdim = std::max<int64_t>(o && o->max_reduced_dim > 0 ? o->max_reduced_dim : std::max(100, 10 * nstates),
                                             3 * nstates);
    int64_t block = o && o->block > 0 ? o->block : 0;
    if (block <= 0) {
        // tangent working set of one transformed trial ~ 16 full doubles arrays
        double per = 16.0 * 8.0 * (double)nov * (double)nov;
        block = std::max<int64_t>(1, std::min<int64_t>(64, (int64_t)(40e9 / per)));
    }
    orbital_differences(ex, eps.d(), no, nv, epsdiff.d());
    std::vector<double> eh(namp);
    CU_CHECK(cudaMemcpyAsync(eh.data(), epsdiff.d(), sizeof(double) * namp, cudaMemcpyDeviceToHost, s));
    CU_CHECK(cudaStreamSynchronize(s));
    std::vector<int64_t> order(namp);
    std::iota(order.begin(), order.end(), 0);
    std::partial_sort(order.begin(), order.begin() + nstates, order.end(),
                      [&](int64_t a, int64_t b) { return eh[a] < eh[b]; });

    DBuf V = dalloc(namp * maxdim, s), AV = dalloc(namp * maxdim, s);
    int64_t dim = 0, nnew = 0;
    DBuf newv = dalloc(namp * std::max<int64_t>(nstates, 1), s);
    if (start) {
        // start vectors supplied (e.g. the converged mixed-precision eigenvectors)
        CU_CHECK(cudaMemcpyAsync(newv.d(), start, sizeof(double) * namp * nstates, cudaMemcpyDeviceToDevice, s));
    } else {
        for (int k = 0; k < nstates; k++)
            unit_vector_kernel<<<grid_for(namp, 256), 256, 0, s>>>(newv.d() + k * namp, namp, order[k]);
    }
    nnew = nstates;
    std::vector<double> omega(nstates, 0.0), prev(nstates, 0.0);
    PrepareScope prepared(*this);
    DBuf G = dalloc(maxdim * maxdim, s), X = dalloc(namp * nstates, s), R = dalloc(namp * nstates, s);
    DBuf proj = dalloc(maxdim * std::max<int64_t>(nstates, 1), s), nrm = dalloc(8, s);
    Geev geev(s);
    int it = 0;
    bool conv = false;
    auto transform = [&](const double *in, double *out, int64_t nv_) {
        for (int64_t c0 = 0; c0 < nv_; c0 += block) {
            int64_t c = std::min(block, nv_ - c0);
            if (side == 0) jacobian(c, in + c0 * namp, out + c0 * namp);
            else jacobian_transpose(c, in + c0 * namp, out + c0 * namp);
        }
    };
    // orthonormalise `count` candidate columns against V and each other; append the survivors.  As in
    // davidson_tool (add_new_trial, davidson_tool_class.F90:342; orthonormalize_trial_vecs, :517) each
    // candidate is normalised first and counts as linearly dependent when less than
    // min(1e-11, 0.1 residual_threshold) of it is left after Gram-Schmidt
    // (cc_es_amplitudes_solver_factory_class.F90:315); eT stops there, this solver drops the candidate.
    const double lindep = std::min(1e-11, 0.1 * rthr);
    auto add_trials = [&](double *cand, int64_t count) {
        for (int64_t k = 0; k < count; k++) {
            double *x = cand + k * namp;
            {
                double c2;
                dot(ex, x, x, namp, nrm.d());
                CU_CHECK(cudaMemcpyAsync(&c2, nrm.d(), sizeof(double), cudaMemcpyDeviceToHost, s));
                CU_CHECK(cudaStreamSynchronize(s));
                if (!(c2 > 0.0)) continue;
                axpby(ex, namp, 1.0 / std::sqrt(c2), x, 0.0, x);
            }
            for (int pass = 0; pass < 2; pass++) {
                if (dim > 0) {
                    // x -= V (V^T x)
                    gemm(ex, true, false, dim, 1, namp, 1.0, V.d(), namp, x, namp, 0.0, proj.d(), dim, false);
                    gemm(ex, false, false, namp, 1, dim, -1.0, V.d(), namp, proj.d(), dim, 1.0, x, namp, false);
                }
            }
            dot(ex, x, x, namp, nrm.d());
            double n2;
            CU_CHECK(cudaMemcpyAsync(&n2, nrm.d(), sizeof(double), cudaMemcpyDeviceToHost, s));
            CU_CHECK(cudaStreamSynchronize(s));
            if (std::sqrt(n2) < lindep || dim >= maxdim) continue;
            axpby(ex, namp, 1.0 / std::sqrt(n2), x, 0.0, V.d() + dim * namp);
            dim++;
        }
    };
    int64_t first_new = 0;
    add_trials(newv.d(), nnew);
    while (it < maxit) {
        it++;
        transform(V.d() + first_new * namp, AV.d() + first_new * namp, dim - first_new);
        // reduced matrix G = V^T A V (column-major dim x dim)
        gemm(ex, true, false, dim, dim, namp, 1.0, V.d(), namp, AV.d(), namp, 0.0, G.d(), dim, false);
        std::vector<std::complex<double>> w;
        std::vector<double> y;
        geev.solve(s, G.d(), dim, w, y);
        std::vector<int64_t> idx(dim);
        std::iota(idx.begin(), idx.end(), 0);
        std::sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return w[a].real() < w[b].real(); });
        std::vector<double> Y(dim * nstates);
        for (int k = 0; k < nstates; k++) {
            omega[k] = w[idx[k]].real();
            for (int64_t r = 0; r < dim; r++) Y[r + dim * k] = y[r + dim * idx[k]];   // real part
        }
        DBuf Yd = dalloc(dim * nstates, s);
        CU_CHECK(cudaMemcpyAsync(Yd.d(), Y.data(), sizeof(double) * dim * nstates, cudaMemcpyHostToDevice, s));
        // Ritz vectors and residuals
        gemm(ex, false, false, namp, nstates, dim, 1.0, V.d(), namp, Yd.d(), dim, 0.0, X.d(), namp, false);
        gemm(ex, false, false, namp, nstates, dim, 1.0, AV.d(), namp, Yd.d(), dim, 0.0, R.d(), namp, false);
        std::vector<double> rn(nstates);
        bool all_conv = true;
        nnew = 0;
        for (int k = 0; k < nstates; k++) {
            double xn2;
            dot(ex, X.d() + k * namp, X.d() + k * namp, namp, nrm.d());
            CU_CHECK(cudaMemcpyAsync(&xn2, nrm.d(), sizeof(double), cudaMemcpyDeviceToHost, s));
            CU_CHECK(cudaStreamSynchronize(s));
            const double xs = 1.0 / std::sqrt(xn2);
            axpby(ex, namp, xs, X.d() + k * namp, 0.0, X.d() + k * namp);           // x <- x / |x|
            axpby(ex, namp, -omega[k], X.d() + k * namp, xs, R.d() + k * namp);     // r = A x - w x
            double r2;
            dot(ex, R.d() + k * namp, R.d() + k * namp, namp, nrm.d());
            CU_CHECK(cudaMemcpyAsync(&r2, nrm.d(), sizeof(double), cudaMemcpyDeviceToHost, s));
            CU_CHECK(cudaStreamSynchronize(s));
            rn[k] = std::sqrt(r2);
            bool ck = rn[k] < rthr && std::fabs(omega[k] - prev[k]) < ethr;
            if (!ck) {
                all_conv = false;
                precondition_kernel<<<grid_for(namp, 256), 256, 0, s>>>(R.d() + k * namp, epsdiff.d(), omega[k], namp,
                                                                       newv.d() + nnew * namp);
                ex.launches++;
                nnew++;
            }
        }
        prev = omega;
        if (all_conv) {
            conv = true;
            break;
        }
        if (dim + nnew > maxdim) {
            // collapse the reduced space onto the current Ritz vectors (davidson_tool restart)
            DBuf cand = dalloc(namp * nstates, s);
            CU_CHECK(cudaMemcpyAsync(cand.d(), X.d(), sizeof(double) * namp * nstates, cudaMemcpyDeviceToDevice, s));
            dim = 0;
            add_trials(cand.d(), nstates);
            transform(V.d(), AV.d(), dim);
        }
        first_new = dim;
        add_trials(newv.d(), nnew);
        if (dim == first_new) break;   // no new directions: stagnated
    }
    if (omega_out) std::copy(omega.begin(), omega.end(), omega_out);
    if (vectors_out)
        CU_CHECK(cudaMemcpyAsync(vectors_out, X.d(), sizeof(double) * namp * nstates, cudaMemcpyDeviceToDevice, s));
    CU_CHECK(cudaStreamSynchronize(s));
    if (iters_out) *iters_out = it;
    return conv ? CCSD_GPU_OK : CCSD_GPU_ENOCONV;
}

// eta of the multiplier equation at the current amplitudes (construct_eta_ccsd)
void Context::eta(double *out) {
    refresh();
    construct_eta(ex, F.d(), g_ovov_const(), no, nv, out);
}

// Multiplier (Lambda) equations  A^T tbar = -eta  by linear Davidson, restating eT's default
// multiplier solver (linear_davidson_solver_class.F90; factory default
// cc_multipliers_solver_factory_class.F90:335-355): Galerkin solve in the trial space built from
// the transpose transformation, orbital-difference preconditioned residuals as new trials.
int Context::multipliers(const ccsd_gpu_davidson_options *o, double *tbar, int32_t *iters_out) {
    REQUIRE(have_t && have_L && have_h, CCSD_GPU_ESTATE, "inputs/amplitudes not set");
    cudaStream_t s = ex.stream;
    const int maxit = o && o->max_iterations > 0 ? o->max_iterations : 100;
    const double rthr = o && o->residual_threshold > 0 ? o->residual_threshold : 1e-6;
    const int64_t maxdim = o && o->max_reduced_dim > 0 ? o->max_reduced_dim : 100;
    orbital_differences(ex, eps.d(), no, nv, epsdiff.d());
    DBuf et = dalloc(namp, s);
    eta(et.d());
    PrepareScope prepared(*this);
    DBuf V = dalloc(namp * maxdim, s), AV = dalloc(namp * maxdim, s), x = dalloc(namp, s), r = dalloc(namp, s);
    DBuf cand = dalloc(namp, s), proj = dalloc(maxdim, s), nrm = dalloc(8, s);
    DBuf G = dalloc(maxdim * maxdim, s), rhs = dalloc(maxdim, s);
    int64_t dim = 0;
    auto host_dot = [&](const double *a, const double *b) {
        dot(ex, a, b, namp, nrm.d());
        double v;
        CU_CHECK(cudaMemcpyAsync(&v, nrm.d(), sizeof(double), cudaMemcpyDeviceToHost, s));
        CU_CHECK(cudaStreamSynchronize(s));
        return v;
    };
    // normalise, Gram-Schmidt twice, drop when less than min(1e-11, 0.1 threshold) remains (as in the
    // eigenvalue solver above)
    const double lindep = std::min(1e-11, 0.1 * rthr);
    auto add_trial = [&](double *c) {
        const double c2 = host_dot(c, c);
        if (!(c2 > 0.0)) return false;
        axpby(ex, namp, 1.0 / std::sqrt(c2), c, 0.0, c);
        for (int pass = 0; pass < 2; pass++)
            if (dim > 0) {
                gemm(ex, true, false, dim, 1, namp, 1.0, V.d(), namp, c, namp, 0.0, proj.d(), dim, false);
                gemm(ex, false, false, namp, 1, dim, -1.0, V.d(), namp, proj.d(), dim, 1.0, c, namp, false);
            }
        double n2 = host_dot(c, c);
        if (std::sqrt(n2) < lindep || dim >= maxdim) return false;
        axpby(ex, namp, 1.0 / std::sqrt(n2), c, 0.0, V.d() + dim * namp);
        jacobian_transpose(1, V.d() + dim * namp, AV.d() + dim * namp);
        dim++;
        return true;
    };
    multiplier_guess(ex, t.d(), no, nv, cand.d());   // set_initial_multipliers_guess_ccsd
    add_trial(cand.d());
    cusolverDnHandle_t hs = nullptr;
    cusolverDnParams_t ps = nullptr;
    SOLVER_CHECK(cusolverDnCreate(&hs));
    SOLVER_CHECK(cusolverDnSetStream(hs, s));
    SOLVER_CHECK(cusolverDnCreateParams(&ps));
    struct Guard {
        cusolverDnHandle_t h;
        cusolverDnParams_t p;
        ~Guard() {
            cusolverDnDestroyParams(p);
            cusolverDnDestroy(h);
        }
    } guard{hs, ps};
    int it = 0;
    bool conv = false;
    while (it < maxit) {
        it++;
        // reduced system (V^T A^T V) y = -V^T eta, solved by LU on the device
        gemm(ex, true, false, dim, dim, namp, 1.0, V.d(), namp, AV.d(), namp, 0.0, G.d(), dim, false);
        gemm(ex, true, false, dim, 1, namp, -1.0, V.d(), namp, et.d(), namp, 0.0, rhs.d(), dim, false);
        DBuf piv(sizeof(int64_t) * dim, s), info(sizeof(int), s);
        size_t db = 0, hb = 0;
        SOLVER_CHECK(cusolverDnXgetrf_bufferSize(hs, ps, dim, dim, CUDA_R_64F, G.d(), dim, CUDA_R_64F, &db, &hb));
        DBuf dw(std::max<size_t>(db, 8), s);
        std::vector<char> hw(std::max<size_t>(hb, 8));
        SOLVER_CHECK(cusolverDnXgetrf(hs, ps, dim, dim, CUDA_R_64F, G.d(), dim, piv.as<int64_t>(), CUDA_R_64F,
                                      dw.as<void>(), db, hw.data(), hb, info.as<int>()));
        SOLVER_CHECK(cusolverDnXgetrs(hs, ps, CUBLAS_OP_N, dim, 1, CUDA_R_64F, G.d(), dim, piv.as<int64_t>(),
                                      CUDA_R_64F, rhs.d(), dim, info.as<int>()));
        int inf = 0;
        CU_CHECK(cudaMemcpyAsync(&inf, info.as<int>(), sizeof(int), cudaMemcpyDeviceToHost, s));
        CU_CHECK(cudaStreamSynchronize(s));
        REQUIRE(inf == 0, CCSD_GPU_ESINGULAR, "reduced multiplier system is singular");
        // x = V y ; r = A^T x + eta = AV y + eta
        gemm(ex, false, false, namp, 1, dim, 1.0, V.d(), namp, rhs.d(), dim, 0.0, x.d(), namp, false);
        CU_CHECK(cudaMemcpyAsync(r.d(), et.d(), sizeof(double) * namp, cudaMemcpyDeviceToDevice, s));
        gemm(ex, false, false, namp, 1, dim, 1.0, AV.d(), namp, rhs.d(), dim, 1.0, r.d(), namp, false);
        const double rn = std::sqrt(host_dot(r.d(), r.d()));
        if (!std::isfinite(rn)) throw Error(CCSD_GPU_ENAN, "non-finite multiplier residual");
        if (rn < rthr) {
            conv = true;
            break;
        }
        if (dim >= maxdim) {
            // restart from the current solution
            CU_CHECK(cudaMemcpyAsync(cand.d(), x.d(), sizeof(double) * namp, cudaMemcpyDeviceToDevice, s));
            dim = 0;
            add_trial(cand.d());
        }
        precondition_kernel<<<grid_for(namp, 256), 256, 0, s>>>(r.d(), epsdiff.d(), 0.0, namp, cand.d());
        ex.launches++;
        if (!add_trial(cand.d())) break;
    }
    CU_CHECK(cudaMemcpyAsync(tbar, x.d(), sizeof(double) * namp, cudaMemcpyDeviceToDevice, s));
    CU_CHECK(cudaStreamSynchronize(s));
    if (iters_out) *iters_out = it;
    return conv ? CCSD_GPU_OK : CCSD_GPU_ENOCONV;
}

}  // namespace ccsd
