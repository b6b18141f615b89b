// Batch executor for independent ground-state solves (ccsd_gpu_solve_gs_batch).
//
// Small systems (o ~ 6..24) leave most of the 148 SMs idle: their contractions are short and every
// solver iteration synchronises the host a few times (residual norm, DIIS status).  Running several
// systems at once, each on its own context and CUDA stream driven by its own host thread, lets the
// kernels of one system fill the gaps of another.  Systems are taken largest-first (o^2 v^4, the
// ladder cost) from a shared counter, so the last ones to start are the short ones.
#include <algorithm>
#include <atomic>
#include <numeric>
#include <thread>
#include <vector>

#include "common.cuh"

extern "C" int ccsd_gpu_solve_gs_batch(int32_t n_systems, const ccsd_gpu_batch_system *systems,
                                       const ccsd_gpu_options *opt, const ccsd_gpu_solver_options *sopt,
                                       int32_t workers, double *energies, int32_t *iterations, int32_t *status) {
    if (n_systems < 0 || (n_systems > 0 && !systems)) return CCSD_GPU_EINVAL;
    if (n_systems == 0) return CCSD_GPU_OK;
    const int nw = std::max(1, std::min<int>(std::min<int>(workers, 64), n_systems));
    std::vector<int> order(n_systems);
    std::iota(order.begin(), order.end(), 0);
    auto cost = [&](int k) {
        const double o = (double)systems[k].n_o, v = (double)systems[k].n_v;
        return o * o * v * v * v * v;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost(a) > cost(b); });
    std::vector<int> rcs(n_systems, CCSD_GPU_OK);
    std::atomic<int> next{0};
    auto work = [&]() {
        while (true) {
            const int i = next.fetch_add(1);
            if (i >= n_systems) break;
            const int k = order[i];
            const ccsd_gpu_batch_system &sys = systems[k];
            void *ctx = nullptr;
            double e = 0.0;
            int32_t it = 0;
            int rc = ccsd_gpu_create(sys.n_o, sys.n_v, sys.n_J, opt, &ctx);
            if (rc == CCSD_GPU_OK) rc = ccsd_gpu_set_cholesky_mo(ctx, sys.L_mo);
            if (rc == CCSD_GPU_OK) rc = ccsd_gpu_set_h_mo(ctx, sys.h_mo, sys.eps, sys.e_hf);
            if (rc == CCSD_GPU_OK) rc = ccsd_gpu_mp2_guess(ctx);
            if (rc == CCSD_GPU_OK) rc = ccsd_gpu_solve_gs(ctx, sopt, &e, &it, nullptr);
            if ((rc == CCSD_GPU_OK || rc == CCSD_GPU_ENOCONV) && sys.t_out) {
                const int r2 = ccsd_gpu_get_amplitudes(ctx, sys.t_out);
                if (rc == CCSD_GPU_OK) rc = r2;
            }
            if (ctx) ccsd_gpu_destroy(ctx);
            rcs[k] = rc;
            if (energies) energies[k] = e;
            if (iterations) iterations[k] = it;
            if (status) status[k] = rc;
        }
    };
    std::vector<std::thread> pool;
    for (int w = 1; w < nw; w++) pool.emplace_back(work);
    work();
    for (auto &th : pool) th.join();
    for (int k = 0; k < n_systems; k++)
        if (rcs[k] != CCSD_GPU_OK) return rcs[k];
    return CCSD_GPU_OK;
}
