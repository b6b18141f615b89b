// extern "C" entry points (include/ccsd_gpu.h): argument checks, host<->device staging,
// and conversion of exceptions into status codes.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>

#include "autotune.cuh"
#include "ccsd.cuh"
#include "mixed_gemm.cuh"
#include "ozaki_gemm.cuh"
#include "ccsd_kernels.cuh"
#include "tensor_ops.cuh"

using ccsd::Context;
using ccsd::Error;

namespace {

thread_local std::string g_create_error;

template <class F>
int guarded(void *ctx, F &&f) {
    if (!ctx) return CCSD_GPU_EINVAL;
    Context *c = static_cast<Context *>(ctx);
    try {
        CU_CHECK(cudaSetDevice(c->device));
        f(*c);
        c->err.clear();
        return CCSD_GPU_OK;
    } catch (const Error &e) {
        c->err = e.what();
        return e.code;
    } catch (const std::bad_alloc &) {
        c->err = "host allocation failed";
        return CCSD_GPU_ENOMEM;
    } catch (const std::exception &e) {
        c->err = e.what();
        return CCSD_GPU_ECUDA;
    }
}

void h2d(Context &c, double *dst, const double *src, int64_t n) {
    REQUIRE(src != nullptr, CCSD_GPU_EINVAL, "null input pointer");
    CU_CHECK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyHostToDevice, c.ex.stream));
}

void d2h(Context &c, double *dst, const double *src, int64_t n) {
    REQUIRE(dst != nullptr, CCSD_GPU_EINVAL, "null output pointer");
    CU_CHECK(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToHost, c.ex.stream));
    CU_CHECK(cudaStreamSynchronize(c.ex.stream));
}

}  // namespace

extern "C" {

int ccsd_gpu_create(int64_t n_o, int64_t n_v, int64_t n_J, const ccsd_gpu_options *opt, void **ctx) {
    if (!ctx) return CCSD_GPU_EINVAL;
    *ctx = nullptr;
    try {
        if (n_o <= 0 || n_v <= 0 || n_J <= 0) throw Error(CCSD_GPU_EINVAL, "dimensions must be positive");
        if (opt && opt->precision != CCSD_GPU_FP64 && opt->precision != CCSD_GPU_MIXED)
            throw Error(CCSD_GPU_EINVAL, "unknown precision");
        *ctx = new Context(n_o, n_v, n_J, opt);
        return CCSD_GPU_OK;
    } catch (const Error &e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::exception &e) {
        g_create_error = e.what();
        return CCSD_GPU_ECUDA;
    }
}

void ccsd_gpu_destroy(void *ctx) {
    if (!ctx) return;
    Context *c = static_cast<Context *>(ctx);
    cudaSetDevice(c->device);
    delete c;
}

const char *ccsd_gpu_last_error(void *ctx) {
    if (!ctx) return g_create_error.c_str();
    return static_cast<Context *>(ctx)->err.c_str();
}

int ccsd_gpu_set_precision(void *ctx, int32_t precision) {
    return guarded(ctx, [&](Context &c) {
        c.set_precision(precision);
    });
}

int ccsd_gpu_set_stream(void *ctx, void *stream) {
    return guarded(ctx, [&](Context &c) {
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
        c.set_stream(static_cast<cudaStream_t>(stream));
    });
}

int ccsd_gpu_synchronize(void *ctx) {
    return guarded(ctx, [&](Context &c) { CU_CHECK(cudaStreamSynchronize(c.ex.stream)); });
}

int ccsd_gpu_set_cholesky_mo(void *ctx, const double *L) {
    return guarded(ctx, [&](Context &c) {
        REQUIRE(L != nullptr, CCSD_GPU_EINVAL, "null L");
        // split (J, n_mo, n_mo) into the four blocks with strided 2-D copies per q
        const int64_t J = c.nJ, nmo = c.nmo, no = c.no, nv = c.nv;
        auto blk = [&](ccsd::DBuf &dst, int64_t p0, int64_t np, int64_t q0, int64_t nq) {
            // dst[J, p, q] <- L[J, p0+p, q0+q]: for each q a contiguous run of J*np
            CU_CHECK(cudaMemcpy2DAsync(dst.d(), sizeof(double) * J * np, L + J * (p0 + nmo * q0),
                                       sizeof(double) * J * nmo, sizeof(double) * J * np, nq,
                                       cudaMemcpyHostToDevice, c.ex.stream));
        };
        blk(c.L_oo, 0, no, 0, no);
        blk(c.L_ov, 0, no, no, nv);
        blk(c.L_vo, no, nv, 0, no);
        blk(c.L_vv, no, nv, no, nv);
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
        c.have_L = true;
        c.have_gov = false;
        c.l_version++;
        if (c.have_h) c.refresh();
    });
}

int ccsd_gpu_set_cholesky_mo_blocks(void *ctx, const double *L_oo, const double *L_ov, const double *L_vo,
                                    const double *L_vv) {
    return guarded(ctx, [&](Context &c) {
        h2d(c, c.L_oo.d(), L_oo, c.nJ * c.no * c.no);
        h2d(c, c.L_ov.d(), L_ov, c.nJ * c.no * c.nv);
        h2d(c, c.L_vo.d(), L_vo, c.nJ * c.nv * c.no);
        h2d(c, c.L_vv.d(), L_vv, c.nJ * c.nv * c.nv);
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
        c.have_L = true;
        c.have_gov = false;
        c.l_version++;
        if (c.have_h) c.refresh();
    });
}

int ccsd_gpu_set_h_mo(void *ctx, const double *h, const double *eps, double e_hf) {
    return guarded(ctx, [&](Context &c) {
        h2d(c, c.h.d(), h, c.nmo * c.nmo);
        h2d(c, c.eps.d(), eps, c.nmo);
        c.set_h_blocks();
        c.e_hf = e_hf;
        ccsd::orbital_differences(c.ex, c.eps.d(), c.no, c.nv, c.epsdiff.d());
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
        c.have_h = true;
        if (c.have_L) c.refresh();
    });
}

int ccsd_gpu_set_amplitudes(void *ctx, const double *t) {
    return guarded(ctx, [&](Context &c) {
        h2d(c, c.t.d(), t, c.namp);
        c.have_t = true;
        c.refresh();
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
    });
}

int ccsd_gpu_get_amplitudes(void *ctx, double *t) {
    return guarded(ctx, [&](Context &c) { d2h(c, t, c.t.d(), c.namp); });
}

int ccsd_gpu_mp2_guess(void *ctx) {
    return guarded(ctx, [&](Context &c) {
        REQUIRE(c.have_L && c.have_h, CCSD_GPU_ESTATE, "Cholesky vectors and h must be set first");
        c.mp2_guess();
        c.refresh();
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
    });
}

int ccsd_gpu_get_fock(void *ctx, double *F) {
    return guarded(ctx, [&](Context &c) { d2h(c, F, c.F.d(), c.nmo * c.nmo); });
}

int ccsd_gpu_energy(void *ctx, double *energy) {
    return guarded(ctx, [&](Context &c) {
        REQUIRE(energy != nullptr, CCSD_GPU_EINVAL, "null output");
        REQUIRE(c.have_t, CCSD_GPU_ESTATE, "amplitudes not set");
        *energy = c.energy();
    });
}

int ccsd_gpu_omega(void *ctx, double *omega) {
    return guarded(ctx, [&](Context &c) {
        REQUIRE(omega != nullptr, CCSD_GPU_EINVAL, "null output");
        ccsd::DBuf om = ccsd::dalloc(c.namp, c.ex.stream);
        c.omega(om.d());
        d2h(c, omega, om.d(), c.namp);
    });
}

int ccsd_gpu_omega_device(void *ctx, double *d_omega) {
    return guarded(ctx, [&](Context &c) {
        REQUIRE(d_omega != nullptr, CCSD_GPU_EINVAL, "null output");
        c.omega(d_omega);
    });
}

int ccsd_gpu_jacobian(void *ctx, int64_t n_vec, const double *c, double *rho) {
    return guarded(ctx, [&](Context &x) {
        REQUIRE(n_vec > 0 && c && rho, CCSD_GPU_EINVAL, "bad jacobian arguments");
        ccsd::DBuf dc = ccsd::dalloc(x.namp * n_vec, x.ex.stream), dr = ccsd::dalloc(x.namp * n_vec, x.ex.stream);
        h2d(x, dc.d(), c, x.namp * n_vec);
        x.jacobian(n_vec, dc.d(), dr.d());
        d2h(x, rho, dr.d(), x.namp * n_vec);
    });
}

int ccsd_gpu_jacobian_transpose(void *ctx, int64_t n_vec, const double *b, double *sigma) {
    return guarded(ctx, [&](Context &x) {
        REQUIRE(n_vec > 0 && b && sigma, CCSD_GPU_EINVAL, "bad transpose arguments");
        ccsd::DBuf db = ccsd::dalloc(x.namp * n_vec, x.ex.stream), ds = ccsd::dalloc(x.namp * n_vec, x.ex.stream);
        h2d(x, db.d(), b, x.namp * n_vec);
        x.jacobian_transpose(n_vec, db.d(), ds.d());
        d2h(x, sigma, ds.d(), x.namp * n_vec);
    });
}

int ccsd_gpu_prepare_jacobian(void *ctx, int32_t side) {
    return guarded(ctx, [&](Context &c) {
        REQUIRE(side >= -1 && side <= 1, CCSD_GPU_EINVAL, "side must be 0 (right), 1 (left) or -1 (release)");
        if (side < 0) c.drop_jacobian();
        else c.prepare_jacobian();
    });
}

int ccsd_gpu_jacobian_device(void *ctx, int64_t n_vec, const double *d_c, double *d_rho) {
    return guarded(ctx, [&](Context &x) {
        REQUIRE(n_vec > 0 && d_c && d_rho, CCSD_GPU_EINVAL, "bad jacobian arguments");
        x.jacobian(n_vec, d_c, d_rho);
    });
}

int ccsd_gpu_jacobian_transpose_device(void *ctx, int64_t n_vec, const double *d_b, double *d_sigma) {
    return guarded(ctx, [&](Context &x) {
        REQUIRE(n_vec > 0 && d_b && d_sigma, CCSD_GPU_EINVAL, "bad transpose arguments");
        x.jacobian_transpose(n_vec, d_b, d_sigma);
    });
}

int ccsd_gpu_vjp(void *ctx, const double *b, double *dt, double *dL, double *dh) {
    return guarded(ctx, [&](Context &x) {
        REQUIRE(b != nullptr, CCSD_GPU_EINVAL, "null cotangent");
        cudaStream_t s = x.ex.stream;
        ccsd::DBuf db = ccsd::dalloc(x.namp, s);
        h2d(x, db.d(), b, x.namp);
        ccsd::DBuf ddt = ccsd::dalloc(x.namp, s);
        ccsd::DBuf ddL = dL ? ccsd::dalloc(x.nJ * x.nmo * x.nmo, s) : ccsd::DBuf();
        ccsd::DBuf ddh = dh ? ccsd::dalloc(x.nmo * x.nmo, s) : ccsd::DBuf();
        x.adjoint(db.d(), ddt.d(), dL ? ddL.d() : nullptr, dh ? ddh.d() : nullptr);
        if (dt) d2h(x, dt, ddt.d(), x.namp);
        if (dL) d2h(x, dL, ddL.d(), x.nJ * x.nmo * x.nmo);
        if (dh) d2h(x, dh, ddh.d(), x.nmo * x.nmo);
    });
}

int ccsd_gpu_one_electron_density(void *ctx, const double *tbar, double *D) {
    return guarded(ctx, [&](Context &x) {
        REQUIRE(tbar != nullptr && D != nullptr, CCSD_GPU_EINVAL, "null multipliers or density");
        cudaStream_t s = x.ex.stream;
        ccsd::DBuf db = ccsd::dalloc(x.namp, s), dD = ccsd::dalloc(x.nmo * x.nmo, s);
        h2d(x, db.d(), tbar, x.namp);
        x.adjoint(db.d(), nullptr, nullptr, dD.d());                   // tbar^T dOmega/dh
        ccsd::density_energy_part(x.ex, dD.d(), x.t.d(), x.no, x.nv);   // + dE/dh
        d2h(x, D, dD.d(), x.nmo * x.nmo);
    });
}

int ccsd_gpu_eom_davidson(void *ctx, int32_t n_states, int32_t side, const ccsd_gpu_davidson_options *opt,
                          double *omega, double *vectors, int32_t *iterations) {
    int status = CCSD_GPU_OK;
    int rc = guarded(ctx, [&](Context &c) {
        REQUIRE(side == 0 || side == 1, CCSD_GPU_EINVAL, "side must be 0 (right) or 1 (left)");
        REQUIRE(omega != nullptr, CCSD_GPU_EINVAL, "null omega");
        ccsd::DBuf dv = vectors ? ccsd::dalloc(c.namp * n_states, c.ex.stream) : ccsd::DBuf();
        const bool start = opt && opt->start_from_vectors;
        REQUIRE(!start || vectors, CCSD_GPU_EINVAL, "start_from_vectors needs the vectors argument");
        if (start) h2d(c, dv.d(), vectors, c.namp * n_states);
        status = c.davidson(n_states, side, opt, omega, vectors ? dv.d() : nullptr, iterations, start ? dv.d() : nullptr);
        if (vectors) d2h(c, vectors, dv.d(), c.namp * n_states);
    });
    if (rc != CCSD_GPU_OK) return rc;
    if (status != CCSD_GPU_OK) static_cast<Context *>(ctx)->err = "Davidson did not converge";
    return status;
}

int ccsd_gpu_construct_eta(void *ctx, double *eta) {
    return guarded(ctx, [&](Context &c) {
        REQUIRE(c.have_t, CCSD_GPU_ESTATE, "amplitudes not set");
        ccsd::DBuf d = ccsd::dalloc(c.namp, c.ex.stream);
        c.eta(d.d());
        d2h(c, eta, d.d(), c.namp);
    });
}

int ccsd_gpu_solve_multipliers(void *ctx, const ccsd_gpu_davidson_options *opt, double *tbar, int32_t *iterations) {
    int status = CCSD_GPU_OK;
    int rc = guarded(ctx, [&](Context &c) {
        ccsd::DBuf d = ccsd::dalloc(c.namp, c.ex.stream);
        status = c.multipliers(opt, d.d(), iterations);
        d2h(c, tbar, d.d(), c.namp);
    });
    if (rc != CCSD_GPU_OK) return rc;
    if (status != CCSD_GPU_OK) static_cast<Context *>(ctx)->err = "multiplier equations did not converge";
    return status;
}

int ccsd_gpu_solve_gs(void *ctx, const ccsd_gpu_solver_options *opt, double *energy, int32_t *iterations,
                      double *history) {
    int status = CCSD_GPU_OK;
    int rc = guarded(ctx, [&](Context &c) { status = c.solve_gs(opt, energy, iterations, history); });
    if (rc != CCSD_GPU_OK) return rc;
    if (status != CCSD_GPU_OK) static_cast<Context *>(ctx)->err = "ground state did not converge";
    return status;
}

int ccsd_gpu_stats(void *ctx, int64_t *kernel_launches, double *gemm_flops) {
    return guarded(ctx, [&](Context &c) {
        if (kernel_launches) *kernel_launches = c.ex.launches;
        if (gemm_flops) *gemm_flops = c.ex.flops;
    });
}

int ccsd_gpu_set_graphs(void *ctx, int32_t on) {
    return guarded(ctx, [&](Context &c) {
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
        c.use_graphs = on != 0;
        if (!c.use_graphs)
            for (auto &G : c.rgraph) G.reset();
    });
}

int ccsd_gpu_set_fp64_digits(void *ctx, int32_t digits, double min_flops) {
    return guarded(ctx, [&](Context &c) {
        REQUIRE(digits == 0 || (digits >= 4 && digits <= 7), CCSD_GPU_EINVAL, "digits must be 0 or 4..7");
        if (digits != c.ex.fp64_digits) c.drop_jacobian();
        c.ex.fp64_digits = digits;
        c.ex.fp64_digits_min_flops = min_flops > 0.0 ? min_flops : 1e10;
    });
}

int ccsd_gpu_digit_gemm_profile(void *ctx, int64_t *launches, double *device_ms, double *int8_ops) {
    return guarded(ctx, [&](Context &c) {
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
        double ms = 0.0, ops = 0.0;
        for (size_t i = 0; i < c.prof.oz_events.size(); i++) {
            float t = 0.f;
            CU_CHECK(cudaEventElapsedTime(&t, c.prof.oz_events[i].first, c.prof.oz_events[i].second));
            ms += t;
            ops += c.prof.oz_ops[i];
        }
        if (launches) *launches = (int64_t)c.prof.oz_events.size();
        if (device_ms) *device_ms = ms;
        if (int8_ops) *int8_ops = ops;
    });
}

int ccsd_gpu_set_fp64_integrals(void *ctx, int32_t resident) {
    return guarded(ctx, [&](Context &c) {
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
        c.f64_resident_on = resident != 0;
        if (!c.f64_resident_on) {
            c.f64_gp.release();
            c.f64_gm.release();
            c.f64_ovvv.release();
            c.f64_version = -1;
            c.cache_epoch++;
        }
    });
}

int ccsd_gpu_set_term_timing(void *ctx, int32_t on) {
    return guarded(ctx, [&](Context &c) {
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
        if (on) c.terms.clear();
        c.terms.on = on != 0;
    });
}

int ccsd_gpu_term_timing_report(void *ctx, char *json, int64_t capacity, int64_t *needed) {
    return guarded(ctx, [&](Context &c) {
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
        std::vector<std::string> order;
        std::vector<std::pair<int64_t, double>> agg;
        for (const auto &m : c.terms.marks) {
            float ms = 0.f;
            CU_CHECK(cudaEventElapsedTime(&ms, m.e0, m.e1));
            size_t k = 0;
            while (k < order.size() && order[k] != m.name) k++;
            if (k == order.size()) {
                order.emplace_back(m.name);
                agg.emplace_back(0, 0.0);
            }
            agg[k].first++;
            agg[k].second += ms;
        }
        std::string out = "{";
        for (size_t k = 0; k < order.size(); k++) {
            char buf[64];
            std::snprintf(buf, sizeof buf, "{\"calls\": %lld, \"ms\": %.4f}", (long long)agg[k].first, agg[k].second);
            out += (k ? ", \"" : "\"") + order[k] + "\": " + buf;
        }
        out += "}";
        if (needed) *needed = (int64_t)out.size() + 1;
        if (json && capacity > 0) {
            const size_t n = std::min<size_t>(out.size(), (size_t)capacity - 1);
            std::memcpy(json, out.data(), n);
            json[n] = '\0';
        }
    });
}

int ccsd_gpu_graph_stats(void *ctx, int64_t *residual_replays, int64_t *tuned_routes) {
    return guarded(ctx, [&](Context &c) {
        if (residual_replays) *residual_replays = c.graph_replays;
        if (tuned_routes) *tuned_routes = ccsd::tune_entries();
    });
}

int ccsd_gpu_set_profiling(void *ctx, int32_t on) {
    return guarded(ctx, [&](Context &c) {
        c.prof.clear();
        c.prof.on = on != 0;
    });
}

int ccsd_gpu_gemm_profile(void *ctx, int64_t *launches, double *device_ms, double *tensor_flops) {
    return guarded(ctx, [&](Context &c) {
        CU_CHECK(cudaStreamSynchronize(c.ex.stream));
        double ms = 0.0, fl = 0.0;
        for (size_t i = 0; i < c.prof.events.size(); i++) {
            float t = 0.f;
            CU_CHECK(cudaEventElapsedTime(&t, c.prof.events[i].first, c.prof.events[i].second));
            ms += t;
            fl += c.prof.flops[i];
        }
        if (launches) *launches = (int64_t)c.prof.events.size();
        if (device_ms) *device_ms = ms;
        if (tensor_flops) *tensor_flops = fl;
    });
}

int ccsd_gpu_selftest_gemm(void *ctx, int32_t mixed, int32_t transA, int32_t transB, int64_t m, int64_t n,
                           int64_t k, double alpha, const double *A, int64_t lda, const double *B, int64_t ldb,
                           double beta, double *C, int64_t ldc) {
    return guarded(ctx, [&](Context &c) {
        REQUIRE(m > 0 && n > 0 && k > 0 && A && B && C, CCSD_GPU_EINVAL, "bad gemm arguments");
        const int64_t na = transA ? lda * m : lda * k, nb = transB ? ldb * k : ldb * n, nc = ldc * n;
        cudaStream_t s = c.ex.stream;
        ccsd::DBuf dA = ccsd::dalloc(na, s), dB = ccsd::dalloc(nb, s), dC = ccsd::dalloc(nc, s);
        h2d(c, dA.d(), A, na);
        h2d(c, dB.d(), B, nb);
        h2d(c, dC.d(), C, nc);
        REQUIRE((mixed >= 0 && mixed <= 2) || (mixed >= 4 && mixed <= 7), CCSD_GPU_EINVAL,
                "mixed must be 0, 1, 2 or 4..7 (int8 digits)");
        if (mixed >= 4) {
            ccsd::ozaki_gemm(c.ex, transA, transB, m, n, k, alpha, dA.d(), lda, dB.d(), ldb, beta, dC.d(), ldc, mixed);
        } else if (mixed) {
            const int planes = c.ex.planes;
            c.ex.planes = mixed == 2 ? 3 : 2;
            try {
                ccsd::mixed_gemm(c.ex, transA, transB, m, n, k, alpha, dA.d(), lda, dB.d(), ldb, beta, dC.d(), ldc);
            } catch (...) {
                c.ex.planes = planes;
                throw;
            }
            c.ex.planes = planes;
        } else ccsd::gemm(c.ex, transA, transB, m, n, k, alpha, dA.d(), lda, dB.d(), ldb, beta, dC.d(), ldc, false);
        d2h(c, C, dC.d(), nc);
        c.check_gemm();
    });
}

int ccsd_gpu_selftest_gemm_stall(void *ctx, int64_t m, int64_t n, int64_t k, int64_t wait_cycles) {
    return guarded(ctx, [&](Context &c) {
        REQUIRE(m > 0 && n > 0 && k > 0 && m <= 4096 && n <= 4096 && k <= 4096, CCSD_GPU_EINVAL,
                "stall test: 0 < m, n, k <= 4096");
        cudaStream_t s = c.ex.stream;
        ccsd::DBuf A = ccsd::dalloc(m * k, s), B = ccsd::dalloc(k * n, s), C = ccsd::dalloc(m * n, s);
        ccsd::fill(c.ex, A.d(), m * k, 1.0);
        ccsd::fill(c.ex, B.d(), k * n, 1.0);
        c.check_gemm();   // an earlier time-out is not this test's
        const int planes = c.ex.planes;
        c.ex.planes = 2;
        c.ex.stall_test = 1;
        c.ex.wait_cycles = wait_cycles;
        try {
            ccsd::mixed_gemm(c.ex, false, false, m, n, k, 1.0, A.d(), m, B.d(), k, 0.0, C.d(), m, 1);
        } catch (...) {
            c.ex.planes = planes;
            c.ex.stall_test = 0;
            c.ex.wait_cycles = 0;
            throw;
        }
        c.ex.planes = planes;
        c.ex.stall_test = 0;
        c.ex.wait_cycles = 0;
        CU_CHECK(cudaStreamSynchronize(s));
        c.check_gemm();   // CCSD_GPU_ETIMEOUT when the withheld stage made the wait run out
    });
}

int ccsd_gpu_mixed_gemm_noalloc(int32_t transA, int32_t transB, int64_t m, int64_t n, int64_t k, double alpha,
                                const double *A, int64_t lda, const double *B, int64_t ldb, double beta, double *C,
                                int64_t ldc, void *stream) {
    try {
        ccsd::mixed_gemm_noalloc(transA != 0, transB != 0, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                 static_cast<cudaStream_t>(stream));
        return CCSD_GPU_OK;
    } catch (const Error &e) {
        g_create_error = e.what();
        return e.code;
    } catch (const std::exception &e) {
        g_create_error = e.what();
        return CCSD_GPU_ECUDA;
    }
}

double ccsd_gpu_omega_flops(void *ctx) {
    if (!ctx) return 0.0;
    return static_cast<Context *>(ctx)->omega_flops();
}

}  // extern "C"
