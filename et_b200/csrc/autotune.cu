// Measured routes for the GEMMs of the mixed-precision path.
//
// Which engine and K-split count serve a product best depends on its shape in ways a fixed rule gets
// wrong at the edges: small products lose to cuBLAS DGEMM once the operand split and the 128 x 256
// tile padding are paid for, and a split count that fills the last wave of the persistent grid for
// one shape leaves it ragged for the next.  The first time a shape is seen (outside stream capture)
// every candidate route runs on the caller's stream into scratch memory and is timed with CUDA
// events; the fastest is kept for the process and, when CCSD_GPU_TUNE_FILE names a file, appended to
// it, so that later processes load the same routes (and so repeat the same rounding).
#include "autotune.cuh"

#include <cfloat>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <mutex>
#include <unordered_map>

#include "mixed_gemm.cuh"

namespace ccsd {

namespace {

struct Table {
    std::mutex mu;
    std::unordered_map<std::string, int> routes;
    bool loaded = false;
    std::string file;
};

Table &table() {
    static Table t;
    return t;
}

// lines "key route" written by earlier processes
void load_locked(Table &t) {
    if (t.loaded) return;
    t.loaded = true;
    const char *f = std::getenv("CCSD_GPU_TUNE_FILE");
    if (!f || !*f) return;
    t.file = f;
    std::ifstream in(t.file);
    std::string key;
    int r = 0;
    while (in >> key >> r) t.routes[key] = r;
}

// x rounded up to one of four steps per octave
int64_t bucket(int64_t x) {
    if (x <= 32) return x;
    const int e = 63 - __builtin_clzll((unsigned long long)x);
    const int64_t step = int64_t(1) << (e - 2);
    return (x + step - 1) / step * step;
}

// one timing at a time: contexts on other host threads keep the fixed rule meanwhile, so their
// kernels are the only ones sharing the GPU with a measurement
std::mutex g_measure_mu;

bool capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &st) != cudaSuccess) return true;
    return st != cudaStreamCaptureStatusNone;
}

bool trace_on() {
    static const bool on = [] {
        const char *e = std::getenv("CCSD_GPU_TRACE");
        return e && std::atoi(e) >= 1;
    }();
    return on;
}

}  // namespace

std::string tune_key(char kind, int64_t m, int64_t n, int64_t k, bool tA, bool tB, const Exec &ex) {
    int dev = 0, nsm = 0;
    CU_CHECK(cudaGetDevice(&dev));
    CU_CHECK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    char buf[192];
    std::snprintf(buf, sizeof buf, "%c/sm%d/p%d/kc%lld/%d%d/%lldx%lldx%lld", kind, nsm, ex.planes,
                  (long long)ex.k_chunk, tA ? 1 : 0, tB ? 1 : 0, (long long)bucket(m), (long long)bucket(n),
                  (long long)bucket(k));
    return buf;
}

int tune_lookup(const std::string &key) {
    Table &t = table();
    std::lock_guard<std::mutex> lock(t.mu);
    load_locked(t);
    auto it = t.routes.find(key);
    return it == t.routes.end() ? -1 : it->second;
}

int64_t tune_entries() {
    Table &t = table();
    std::lock_guard<std::mutex> lock(t.mu);
    return (int64_t)t.routes.size();
}

int tune_measure(Exec &ex, const std::string &key, const std::vector<int> &routes,
                 const std::function<void(int)> &run) {
    if (routes.empty() || capturing(ex.stream)) return -1;
    std::unique_lock<std::mutex> measuring(g_measure_mu, std::try_to_lock);
    if (!measuring.owns_lock()) return -1;
    {
        // another thread may have stored this shape since the caller looked it up
        const int known = tune_lookup(key);
        if (known >= 0) return known;
    }
    // the candidate runs leave the caller's counters and profile as they were
    const double flops0 = ex.flops;
    const int64_t launches0 = ex.launches;
    GemmProfile *prof = ex.prof;
    ex.prof = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CU_CHECK(cudaEventCreate(&e0));
    CU_CHECK(cudaEventCreate(&e1));
    int best = -1;
    float best_ms = FLT_MAX;
    std::string why;
    for (int r : routes) {
        try {
            run(r);   // first use: allocations, kernel attributes, caches
            CU_CHECK(cudaEventRecord(e0, ex.stream));
            run(r);
            CU_CHECK(cudaEventRecord(e1, ex.stream));
            CU_CHECK(cudaEventSynchronize(e1));
            float ms = 0.f;
            CU_CHECK(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < 2.0f) {
                // short products: average over a few more runs
                const int reps = std::max(2, std::min(8, (int)(4.0f / std::max(ms, 0.05f))));
                CU_CHECK(cudaEventRecord(e0, ex.stream));
                for (int i = 0; i < reps; i++) run(r);
                CU_CHECK(cudaEventRecord(e1, ex.stream));
                CU_CHECK(cudaEventSynchronize(e1));
                CU_CHECK(cudaEventElapsedTime(&ms, e0, e1));
                ms /= reps;
            }
            if (ms < best_ms) {
                best_ms = ms;
                best = r;
            }
        } catch (const Error &e) {
            // a route that cannot run here (its scratch does not fit, say) is skipped
            why = e.what();
            cudaGetLastError();
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ex.flops = flops0;
    ex.launches = launches0;
    ex.prof = prof;
    REQUIRE(best >= 0, CCSD_GPU_ECUDA, "autotune: no route of " + key + " ran: " + why);
    Table &t = table();
    {
        std::lock_guard<std::mutex> lock(t.mu);
        load_locked(t);
        t.routes[key] = best;
        if (!t.file.empty()) {
            std::ofstream out(t.file, std::ios::app);
            out << key << ' ' << best << '\n';
        }
    }
    if (trace_on()) std::fprintf(stderr, "ccsd_gpu tune %s -> route %d (%.3f ms)\n", key.c_str(), best, best_ms);
    return best;
}

void tc_gemm_f64_tuned(Exec &ex, const __nv_bfloat16 *A, int64_t Mp, const __nv_bfloat16 *B, int64_t Np, int64_t Kp,
                       int64_t m, int64_t n, int64_t k_true, double alpha, double beta, double *C, int64_t ldc,
                       int fixed) {
    int splits = fixed;
    if (ex.autotune) {
        const std::string key = tune_key('p', m, n, Kp, false, true, ex);
        int r = tune_lookup(key);
        if (r < 0) {
            DBuf scratch = dalloc(m * n, ex.stream);
            r = tune_measure(ex, key, tc_split_candidates(m, n, Kp, ex.planes), [&](int s) {
                tc_gemm_f64(ex, A, Mp, B, Np, Kp, m, n, k_true, alpha, 0.0, scratch.d(), m, s);
            });
        }
        if (r >= 1) splits = r;
    }
    tc_gemm_f64(ex, A, Mp, B, Np, Kp, m, n, k_true, alpha, beta, C, ldc, splits);
}

}  // namespace ccsd
