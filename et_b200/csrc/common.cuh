// Shared infrastructure of libccsd_gpu: errors, device buffers, tensor views.
#pragma once

#include <cuda_runtime.h>
#include <cublas_v2.h>
#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ccsd_gpu.h"

namespace ccsd {

struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define CU_CHECK(x)                                                                        \
    do {                                                                                   \
        cudaError_t err__ = (x);                                                           \
        if (err__ != cudaSuccess) {                                                        \
            int code__ = (err__ == cudaErrorMemoryAllocation) ? CCSD_GPU_ENOMEM : CCSD_GPU_ECUDA; \
            throw ::ccsd::Error(code__, std::string(#x) + ": " + cudaGetErrorString(err__) + \
                                " (" __FILE__ ":" + std::to_string(__LINE__) + ")");       \
        }                                                                                  \
    } while (0)

#define BLAS_CHECK(x)                                                                      \
    do {                                                                                   \
        cublasStatus_t st__ = (x);                                                         \
        if (st__ != CUBLAS_STATUS_SUCCESS)                                                 \
            throw ::ccsd::Error(CCSD_GPU_ECUDA, std::string(#x) + ": cublas status " +     \
                                std::to_string((int)st__) + " (" __FILE__ ":" +           \
                                std::to_string(__LINE__) + ")");                           \
    } while (0)

#define REQUIRE(cond, code, msg)                                                           \
    do {                                                                                   \
        if (!(cond)) throw ::ccsd::Error(code, msg);                                       \
    } while (0)

// Stream-ordered device buffer (cudaMallocAsync from the device's default pool).
class DBuf {
  public:
    DBuf() = default;
    DBuf(size_t bytes, cudaStream_t s) { alloc(bytes, s); }
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    DBuf(DBuf &&o) noexcept { *this = std::move(o); }
    DBuf &operator=(DBuf &&o) noexcept {
        if (this != &o) {
            release();
            p_ = o.p_;
            bytes_ = o.bytes_;
            s_ = o.s_;
            o.p_ = nullptr;
            o.bytes_ = 0;
        }
        return *this;
    }
    ~DBuf() { release(); }
    void alloc(size_t bytes, cudaStream_t s) {
        release();
        s_ = s;
        bytes_ = bytes;
        if (bytes) CU_CHECK(cudaMallocAsync(&p_, bytes, s));
    }
    void release() noexcept {
        if (p_) cudaFreeAsync(p_, s_);
        p_ = nullptr;
        bytes_ = 0;
    }
    template <class T = double> T *as() const { return static_cast<T *>(p_); }
    double *d() const { return static_cast<double *>(p_); }
    size_t bytes() const { return bytes_; }
    explicit operator bool() const { return p_ != nullptr; }

  private:
    void *p_ = nullptr;
    size_t bytes_ = 0;
    cudaStream_t s_ = nullptr;
};

inline DBuf dalloc(int64_t n, cudaStream_t s) { return DBuf(size_t(n) * sizeof(double), s); }

// A strided view of up to 6 dimensions (element strides, column-major by default).
struct TV {
    double *p = nullptr;
    int nd = 0;
    int64_t n[6] = {0, 0, 0, 0, 0, 0};
    int64_t s[6] = {0, 0, 0, 0, 0, 0};
    int64_t size() const {
        int64_t t = 1;
        for (int k = 0; k < nd; k++) t *= n[k];
        return t;
    }
};

inline TV tv(const double *p, std::initializer_list<int64_t> dims) {
    TV v;
    v.p = const_cast<double *>(p);
    int64_t st = 1;
    for (int64_t d : dims) {
        v.n[v.nd] = d;
        v.s[v.nd] = st;
        st *= d;
        v.nd++;
    }
    return v;
}

enum class Prec { FP64, MIXED };

// CUDA-event timing of the tensor-core GEMM launches (enabled on request).
struct GemmProfile {
    bool on = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    std::vector<double> flops;    // tensor flops issued per launch (3 products x 2mnk)
    // the int8 digit GEMM of FP64-accurate evaluations: its launches and int8 ops issued
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> oz_events;
    std::vector<double> oz_ops;
    void clear() {
        for (auto *v : {&events, &oz_events})
            for (auto &e : *v) {
                cudaEventDestroy(e.first);
                cudaEventDestroy(e.second);
            }
        events.clear();
        flops.clear();
        oz_events.clear();
        oz_ops.clear();
    }
    ~GemmProfile() { clear(); }
};

// Execution environment handed to the tensor kernels.
// Device time per named term, eT's timing labels (timings_class.F90:20-80 writes them to
// eT.timing.out): a pair of CUDA events on the context's stream around each term while `on`.
struct TermLog {
    bool on = false;
    struct Mark {
        const char *name;   // a string literal
        cudaEvent_t e0, e1;
    };
    std::vector<Mark> marks;
    void clear() {
        for (auto &m : marks) {
            cudaEventDestroy(m.e0);
            cudaEventDestroy(m.e1);
        }
        marks.clear();
    }
    ~TermLog() { clear(); }
};

struct Exec {
    cudaStream_t stream = nullptr;
    cublasHandle_t blas = nullptr;
    Prec prec = Prec::FP64;
    double mixed_min_flops = 2e9;
    int planes = 2;              // split-bf16 planes of a mixed GEMM: 2 = bf16x3, 3 = bf16x6
    int64_t k_chunk = 4096;      // K elements a tensor-core accumulator sums before FP64 takes over (<= 0: all)
    bool autotune = false;       // mixed GEMM routes (DGEMM or tensor cores, K splits) from measurement
    double flops = 0.0;          // algorithmic flops issued (counted by contract())
    int64_t launches = 0;        // kernels of this library launched
    GemmProfile *prof = nullptr;
    TermLog *terms = nullptr;
    int *gemm_err = nullptr;     // device error word of this caller's tensor-core GEMMs (one per context)
    long long wait_cycles = 0;   // bound of the GEMM's barrier waits (<= 0: the default, ~2 s)
    int stall_test = 0;          // diagnostics only: the next GEMMs withhold one stage of loads
    // FP64 products of at least 1e10 flops (and 256 in every dimension) run on the int8 tensor
    // cores with this many 7-bit digits per operand (ozaki_gemm); 0 = cuBLAS DGEMM
    int fp64_digits = 0;
    double fp64_digits_min_flops = 1e10;
    // digits of the first-order (FP64) terms inside a mixed-precision residual (0: cuBLAS DGEMM)
    int mixed_fp64_digits = 6;
    // grow-only scratch of the digit GEMM (digit planes and exponents), owned by the context: the
    // multi-GB planes are neither allocated nor freed per product
    DBuf *digit_arena = nullptr;
};

// Times the enclosing scope as one term of ex.terms (nothing happens unless the log is on, and
// nothing is recorded while the stream is being captured into a graph).
class TermTimer {
  public:
    TermTimer(Exec &ex, const char *name) : ex_(ex) {
        if (!ex.terms || !ex.terms->on) return;
        cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(ex.stream, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) return;
        mark_.name = name;
        if (cudaEventCreate(&mark_.e0) != cudaSuccess) return;
        if (cudaEventCreate(&mark_.e1) != cudaSuccess) {
            cudaEventDestroy(mark_.e0);
            return;
        }
        cudaEventRecord(mark_.e0, ex.stream);
        active_ = true;
    }
    ~TermTimer() {
        if (!active_) return;
        cudaEventRecord(mark_.e1, ex_.stream);
        ex_.terms->marks.push_back(mark_);
    }
    TermTimer(const TermTimer &) = delete;
    TermTimer &operator=(const TermTimer &) = delete;

  private:
    Exec &ex_;
    TermLog::Mark mark_{};
    bool active_ = false;
};

}  // namespace ccsd
