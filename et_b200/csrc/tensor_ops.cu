// Tensor primitives: strided permutations (smem-tiled when the fastest index changes),
// GEMM-backed contractions, packed-doubles conversions and deterministic reductions.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>

#include "autotune.cuh"
#include "mixed_gemm.cuh"
#include "ozaki_gemm.cuh"
#include "tensor_ops.cuh"

namespace ccsd {

namespace {

constexpr int MAXD = 6;

struct PermArgs {
    int nd;
    int64_t n[MAXD];
    int64_t si[MAXD];
    int64_t so[MAXD];
};

// One output element per thread; dims are ordered by output stride (dim 0 fastest).
__global__ void permute_simple_kernel(PermArgs a, int64_t total, double alpha, const double *__restrict__ in,
                                      double beta, double *__restrict__ out) {
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = idx, oi = 0, oo = 0;
#pragma unroll
        for (int d = 0; d < MAXD; d++) {
            if (d < a.nd) {
                int64_t q = r / a.n[d];
                int64_t i = r - q * a.n[d];
                r = q;
                oi += i * a.si[d];
                oo += i * a.so[d];
            }
        }
        double v = alpha * in[oi];
        if (beta != 0.0) v += beta * out[oo];
        out[oo] = v;
    }
}

// Rows of the output-fastest dim (dim 0, at least 16 long): a warp takes one row, so the int64
// div/mod chain that locates a row in the other dims runs once per row instead of once per element,
// and both sides stream along dim 0 (this kernel serves permutations whose input-fastest dim is dim
// 0 as well, or whose other dims are too short for the tiled transpose).
__global__ void permute_rows_kernel(PermArgs a, int64_t nrows, double alpha, const double *__restrict__ in,
                                    double beta, double *__restrict__ out) {
    const int64_t n0 = a.n[0], si0 = a.si[0], so0 = a.so[0];
    for (int64_t row = (int64_t)blockIdx.x * blockDim.y + threadIdx.y; row < nrows;
         row += (int64_t)gridDim.x * blockDim.y) {
        int64_t r = row, oi = 0, oo = 0;
#pragma unroll
        for (int d = 1; d < MAXD; d++) {
            if (d < a.nd) {
                const int64_t q = r / a.n[d];
                const int64_t i = r - q * a.n[d];
                r = q;
                oi += i * a.si[d];
                oo += i * a.so[d];
            }
        }
        const double *src = in + oi;
        double *dst = out + oo;
        if (beta == 0.0) {
            for (int64_t i0 = threadIdx.x; i0 < n0; i0 += 32) dst[i0 * so0] = alpha * src[i0 * si0];
        } else {
            for (int64_t i0 = threadIdx.x; i0 < n0; i0 += 32) dst[i0 * so0] = alpha * src[i0 * si0] + beta * dst[i0 * so0];
        }
    }
}

// 32x32 tile over (p = input-fastest dim, q = output-fastest dim); the remaining dims
// are flattened into the z loop.  Dims 2.. of `a` are the batch dims.
__global__ void permute_tiled_kernel(PermArgs a, int64_t nbatch, double alpha, const double *__restrict__ in,
                                     double beta, double *__restrict__ out) {
    __shared__ double tile[32][33];
    const int64_t np = a.n[0], nq = a.n[1];
    const int64_t p0 = (int64_t)blockIdx.x * 32, q0 = (int64_t)blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int64_t b = blockIdx.z; b < nbatch; b += gridDim.z) {
        int64_t r = b, bi = 0, bo = 0;
        for (int d = 2; d < a.nd; d++) {
            int64_t q = r / a.n[d];
            int64_t i = r - q * a.n[d];
            r = q;
            bi += i * a.si[d];
            bo += i * a.so[d];
        }
        for (int k = ty; k < 32; k += 8) {
            int64_t p = p0 + tx, q = q0 + k;
            if (p < np && q < nq) tile[k][tx] = in[bi + p * a.si[0] + q * a.si[1]];
        }
        __syncthreads();
        for (int k = ty; k < 32; k += 8) {
            int64_t q = q0 + tx, p = p0 + k;
            if (p < np && q < nq) {
                int64_t o = bo + p * a.so[0] + q * a.so[1];
                double v = alpha * tile[tx][k];
                if (beta != 0.0) v += beta * out[o];
                out[o] = v;
            }
        }
        __syncthreads();
    }
}

int grid_for(int64_t total, int block) {
    int64_t g = (total + block - 1) / block;
    return (int)std::min<int64_t>(std::max<int64_t>(g, 1), 148 * 32);
}

}  // namespace

namespace {
// CCSD_GPU_TRACE=2: every permutation on stderr, tagged with the contraction that asked for it
thread_local const char *g_perm_tag = nullptr;
int trace_level() {
    static const int level = [] {
        const char *e = std::getenv("CCSD_GPU_TRACE");
        return e ? std::atoi(e) : 0;
    }();
    return level;
}
// CCSD_GPU_TRACE=3 adds the host time spent inside each contraction call: a call that blocks (an
// allocation that grows the pool, a synchronising library call) shows up as a long one
struct PermTag {
    const char *prev;
    std::chrono::steady_clock::time_point t0;
    explicit PermTag(const char *t) : prev(g_perm_tag), t0(std::chrono::steady_clock::now()) { g_perm_tag = t; }
    ~PermTag() {
        if (trace_level() >= 3)
            std::fprintf(stderr, "ccsd_gpu   [%s] host %.3f ms\n", g_perm_tag,
                         std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
        g_perm_tag = prev;
    }
};
}  // namespace

void permute_add(Exec &ex, double alpha, const TV &in, double beta, const TV &out) {
    REQUIRE(in.nd == out.nd, CCSD_GPU_EINVAL, "permute_add: rank mismatch");
    if (trace_level() >= 2) {
        std::string d;
        for (int k = 0; k < in.nd; k++)
            d += " " + std::to_string(in.n[k]) + ":" + std::to_string(in.s[k]) + "->" + std::to_string(out.s[k]);
        std::fprintf(stderr, "ccsd_gpu permute [%s] %.1f MB beta %g dims%s\n", g_perm_tag ? g_perm_tag : "direct",
                     8e-6 * (double)in.size(), beta, d.c_str());
    }
    // drop unit dims
    std::vector<int> dims;
    for (int d = 0; d < in.nd; d++) {
        REQUIRE(in.n[d] == out.n[d], CCSD_GPU_EINVAL, "permute_add: extent mismatch");
        if (in.n[d] > 1) dims.push_back(d);
    }
    int64_t total = in.size();
    if (total == 0) return;
    PermArgs a{};
    if (dims.empty()) dims.push_back(0);
    // order by output stride
    std::sort(dims.begin(), dims.end(), [&](int x, int y) { return out.s[x] < out.s[y]; });
    int q = dims[0];                                       // output-fastest
    int p = *std::min_element(dims.begin(), dims.end(), [&](int x, int y) { return in.s[x] < in.s[y]; });
    if (p != q && in.n[p] >= 8 && in.n[q] >= 8) {
        a.nd = (int)dims.size();
        a.n[0] = in.n[p];
        a.si[0] = in.s[p];
        a.so[0] = out.s[p];
        a.n[1] = in.n[q];
        a.si[1] = in.s[q];
        a.so[1] = out.s[q];
        int k = 2;
        int64_t nb = 1;
        for (int d : dims)
            if (d != p && d != q) {
                a.n[k] = in.n[d];
                a.si[k] = in.s[d];
                a.so[k] = out.s[d];
                nb *= in.n[d];
                k++;
            }
        dim3 grid((unsigned)((a.n[0] + 31) / 32), (unsigned)((a.n[1] + 31) / 32),
                  (unsigned)std::min<int64_t>(nb, 65535));
        permute_tiled_kernel<<<grid, dim3(32, 8), 0, ex.stream>>>(a, nb, alpha, in.p, beta, out.p);
    } else {
        a.nd = (int)dims.size();
        for (size_t k = 0; k < dims.size(); k++) {
            a.n[k] = in.n[dims[k]];
            a.si[k] = in.s[dims[k]];
            a.so[k] = out.s[dims[k]];
        }
        if (a.n[0] >= 16) {
            const int64_t nrows = total / a.n[0];
            const int blocks = (int)std::min<int64_t>((nrows + 7) / 8, 148 * 64);
            permute_rows_kernel<<<blocks, dim3(32, 8), 0, ex.stream>>>(a, nrows, alpha, in.p, beta, out.p);
        } else {
            permute_simple_kernel<<<grid_for(total, 256), 256, 0, ex.stream>>>(a, total, alpha, in.p, beta, out.p);
        }
    }
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// GEMM dispatch
// ---------------------------------------------------------------------------

namespace {

// Route of an m x n x k product: tensor cores (mixed, with `splits` K splits; -1 = the fixed rule's
// count) or the FP64 engines.  known = false: the product is to be timed first (autotune on, a shape
// not seen before); `key` then names it.
struct Route {
    bool known = true, mixed = false;
    int splits = -1;
    std::string key;
};

// fixed rule: the tensor-core tile is 128 x 256 x 64, so skinny products stay on the FP64 pipe
Route fixed_route(const Exec &ex, int64_t m, int64_t n, int64_t k, double fl, bool allow_mixed) {
    Route r;
    const bool tc_ok = allow_mixed && ex.prec == Prec::MIXED && k >= 16;
    r.mixed = tc_ok && fl >= ex.mixed_min_flops && (ex.mixed_min_flops <= 1 || (m >= 64 && n >= 64 && k >= 64));
    return r;
}

Route lookup_route(Exec &ex, bool transA, bool transB, int64_t m, int64_t n, int64_t k, double fl, bool allow_mixed) {
    Route r;
    const bool tc_ok = allow_mixed && ex.prec == Prec::MIXED && k >= 16;
    if (tc_ok && ex.autotune) {
        // measured route (0 = DGEMM, s >= 1 = tensor cores with s K-splits) for products big enough
        // to be worth timing
        if (fl < 5e7 || m < 16 || n < 16) {
            r.splits = 0;
            return r;
        }
        r.key = tune_key('g', m, n, k, transA, transB, ex);
        const int route = tune_lookup(r.key);
        if (route < 0) {
            r.known = false;
            return r;
        }
        r.mixed = route > 0;
        r.splits = route;
        return r;
    }
    return fixed_route(ex, m, n, k, fl, allow_mixed);
}

}  // namespace

void gemm(Exec &ex, bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha, const double *A,
          int64_t lda, const double *B, int64_t ldb, double beta, double *C, int64_t ldc, bool allow_mixed) {
    if (m == 0 || n == 0) return;
    double fl = 2.0 * double(m) * double(n) * double(k);
    ex.flops += fl;
    Route rt = lookup_route(ex, transA, transB, m, n, k, fl, allow_mixed);
    if (!rt.known) {
        std::vector<int> routes;
        if (fl <= 4e11) routes.push_back(0);   // larger products never favour FP64
        for (int sp : tc_split_candidates(m, n, k, ex.planes)) routes.push_back(sp);
        DBuf scratch = dalloc(m * n, ex.stream);
        const int route = tune_measure(ex, rt.key, routes, [&](int r) {
            if (r == 0) {
                const double zero = 0.0;
                BLAS_CHECK(cublasDgemm_64(ex.blas, transA ? CUBLAS_OP_T : CUBLAS_OP_N,
                                          transB ? CUBLAS_OP_T : CUBLAS_OP_N, m, n, k, &alpha, A, lda, B, ldb,
                                          &zero, scratch.d(), m));
            } else {
                mixed_gemm(ex, transA, transB, m, n, k, alpha, A, lda, B, ldb, 0.0, scratch.d(), m, r);
            }
        });
        if (route < 0) {
            // not timed now (another thread is timing, or the stream is being captured): the fixed rule
            rt = fixed_route(ex, m, n, k, fl, allow_mixed);
        } else {
            rt.known = true;
            rt.mixed = route > 0;
            rt.splits = route;
        }
    }
    const bool mixed = rt.mixed;
    const int route = rt.splits;
    if (trace_level() >= 2)
        std::fprintf(stderr, "ccsd_gpu gemm [%s] %s m %lld n %lld k %lld  %.3g flop  splits %d\n",
                     g_perm_tag ? g_perm_tag : "direct", mixed ? "bf16x3" : "fp64", (long long)m, (long long)n,
                     (long long)k, fl, route);
    if (mixed) {
        mixed_gemm(ex, transA, transB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, route);
        return;
    }
    if (ex.fp64_digits > 0 && fl >= ex.fp64_digits_min_flops &&
        (ex.fp64_digits_min_flops <= 1 || (m >= 256 && n >= 256 && k >= 512))) {
        ozaki_gemm(ex, transA, transB, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, ex.fp64_digits);
        return;
    }
    BLAS_CHECK(cublasDgemm_64(ex.blas, transA ? CUBLAS_OP_T : CUBLAS_OP_N, transB ? CUBLAS_OP_T : CUBLAS_OP_N, m,
                              n, k, &alpha, A, lda, B, ldb, &beta, C, ldc));
}

void gemm_batched_f64(Exec &ex, bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha,
                      const double *A, int64_t lda, int64_t strideA, const double *B, int64_t ldb, int64_t strideB,
                      double beta, double *C, int64_t ldc, int64_t strideC, int64_t batch) {
    if (m == 0 || n == 0 || batch == 0) return;
    ex.flops += 2.0 * double(m) * double(n) * double(k) * double(batch);
    BLAS_CHECK(cublasDgemmStridedBatched_64(ex.blas, transA ? CUBLAS_OP_T : CUBLAS_OP_N,
                                            transB ? CUBLAS_OP_T : CUBLAS_OP_N, m, n, k, &alpha, A, lda, strideA, B,
                                            ldb, strideB, &beta, C, ldc, strideC, batch));
}

// ---------------------------------------------------------------------------
// contract()
// ---------------------------------------------------------------------------

namespace {

struct LabelInfo {
    int64_t n = 1;
    int dA = -1, dB = -1, dC = -1;
};

// Is `v` (dims given by `order1` then `order2`) a column-major matrix [group1][group2]?
// Returns the leading dimension in *ld.
bool groupable(const TV &v, const std::vector<int> &g1, const std::vector<int> &g2, int64_t *ld) {
    int64_t expect = 1;
    for (int d : g1) {
        if (v.n[d] == 1) continue;
        if (v.s[d] != expect) return false;
        expect *= v.n[d];
    }
    int64_t lead = -1, exp2 = -1;
    for (int d : g2) {
        if (v.n[d] == 1) continue;
        if (lead < 0) {
            lead = v.s[d];
            if (lead < expect) return false;
            exp2 = lead * v.n[d];
        } else {
            if (v.s[d] != exp2) return false;
            exp2 *= v.n[d];
        }
    }
    *ld = lead < 0 ? std::max<int64_t>(expect, 1) : lead;
    return true;
}

std::vector<char> natural_order(const TV &v, const std::vector<char> &labels, const std::map<char, LabelInfo> &info,
                                int which) {
    std::vector<char> out = labels;
    std::stable_sort(out.begin(), out.end(), [&](char x, char y) {
        const LabelInfo &a = info.at(x), &b = info.at(y);
        int da = which == 0 ? a.dA : which == 1 ? a.dB : a.dC;
        int db = which == 0 ? b.dA : which == 1 ? b.dB : b.dC;
        return v.s[da] < v.s[db];
    });
    return out;
}

std::vector<int> dims_of(const std::vector<char> &labels, const std::map<char, LabelInfo> &info, int which) {
    std::vector<int> d;
    for (char c : labels) {
        const LabelInfo &li = info.at(c);
        d.push_back(which == 0 ? li.dA : which == 1 ? li.dB : li.dC);
    }
    return d;
}

int64_t prod(const std::vector<char> &labels, const std::map<char, LabelInfo> &info) {
    int64_t p = 1;
    for (char c : labels) p *= info.at(c).n;
    return p;
}

// Contiguous copy of v with dims reordered as [g1 labels][g2 labels].
TV make_contiguous(Exec &ex, const TV &v, const std::vector<int> &g1, const std::vector<int> &g2, DBuf &buf) {
    buf = dalloc(v.size(), ex.stream);
    TV dst;
    dst.p = buf.d();
    dst.nd = v.nd;
    int64_t st = 1;
    for (int k = 0; k < v.nd; k++) dst.n[k] = v.n[k];
    for (int d : g1) {
        dst.s[d] = st;
        st *= v.n[d];
    }
    for (int d : g2) {
        dst.s[d] = st;
        st *= v.n[d];
    }
    permute_add(ex, 1.0, v, 0.0, dst);
    return dst;
}

// v as a GEMM operand gather: rows over the dims `rows`, K over the dims `ks` (each in the order
// given, first fastest; unit dims dropped).  False when a group spans more than four dims.
bool gather_view(const TV &v, const std::vector<int> &rows, const std::vector<int> &ks, SplitView *out) {
    SplitView g{};
    g.p = v.p;
    for (int d : rows) {
        if (v.n[d] == 1) continue;
        if (g.nr == 4) return false;
        g.rn[g.nr] = v.n[d];
        g.rs[g.nr++] = v.s[d];
    }
    for (int d : ks) {
        if (v.n[d] == 1) continue;
        if (g.nk == 4) return false;
        g.kn[g.nk] = v.n[d];
        g.ks[g.nk++] = v.s[d];
    }
    if (g.nr == 0) g.rn[g.nr++] = 1;   // a single row (stride unused)
    if (g.nk == 0) g.kn[g.nk++] = 1;
    *out = g;
    return true;
}

}  // namespace

void contract(Exec &ex, const char *spec, double alpha, const TV &A, const TV &B, double beta, const TV &C) {
    PermTag tag(spec);
    std::string s(spec);
    size_t comma = s.find(','), arrow = s.find("->");
    REQUIRE(comma != std::string::npos && arrow != std::string::npos, CCSD_GPU_EINVAL, "contract: bad spec");
    std::string la = s.substr(0, comma), lb = s.substr(comma + 1, arrow - comma - 1), lc = s.substr(arrow + 2);
    REQUIRE((int)la.size() == A.nd && (int)lb.size() == B.nd && (int)lc.size() == C.nd, CCSD_GPU_EINVAL,
            std::string("contract: rank mismatch in ") + spec);
    std::map<char, LabelInfo> info;
    for (int d = 0; d < A.nd; d++) {
        info[la[d]].dA = d;
        info[la[d]].n = A.n[d];
    }
    for (int d = 0; d < B.nd; d++) {
        auto &li = info[lb[d]];
        REQUIRE(li.dA < 0 || li.n == B.n[d], CCSD_GPU_EINVAL, std::string("contract: extent mismatch in ") + spec);
        li.dB = d;
        li.n = B.n[d];
    }
    for (int d = 0; d < C.nd; d++) {
        auto &li = info[lc[d]];
        REQUIRE(li.dA >= 0 || li.dB >= 0, CCSD_GPU_EINVAL, std::string("contract: free output label in ") + spec);
        REQUIRE(li.n == C.n[d], CCSD_GPU_EINVAL, std::string("contract: output extent mismatch in ") + spec);
        li.dC = d;
    }
    std::vector<char> K, M, N;
    for (auto &kv : info) {
        const LabelInfo &li = kv.second;
        int cnt = (li.dA >= 0) + (li.dB >= 0) + (li.dC >= 0);
        REQUIRE(cnt == 2, CCSD_GPU_EINVAL, std::string("contract: label must appear exactly twice in ") + spec);
        if (li.dA >= 0 && li.dB >= 0) K.push_back(kv.first);
        else if (li.dA >= 0) M.push_back(kv.first);
        else N.push_back(kv.first);
    }
    const int64_t mK = prod(K, info), mM = prod(M, info), mN = prod(N, info);
    if (mM == 0 || mN == 0) return;

    // label orders: M/N from C where possible, K from A
    std::vector<char> oM = natural_order(C, M, info, 2), oN = natural_order(C, N, info, 2);
    std::vector<char> oK = natural_order(A, K, info, 0);
    {
        std::vector<char> bK = natural_order(B, K, info, 1);
        int64_t ld;
        // prefer B's K order when B is the bigger operand and already groupable with it
        if (B.size() > A.size() && (groupable(B, dims_of(bK, info, 1), dims_of(oN, info, 1), &ld) ||
                                    groupable(B, dims_of(oN, info, 1), dims_of(bK, info, 1), &ld)))
            oK = bK;
    }
    DBuf bufA, bufB, bufC;
    TV Au = A, Bu = B;
    bool tA, tB;
    int64_t lda, ldb, ldc;
    // an operand whose indices are not two contiguous groups is reordered into a copy, unless the
    // product goes to the tensor cores, whose operand split gathers it from its own layout
    bool packA = false, packB = false;
    const auto aK = dims_of(oK, info, 0), aM = dims_of(oM, info, 0);
    const auto bK = dims_of(oK, info, 1), bN = dims_of(oN, info, 1);
    if (groupable(A, aM, aK, &lda)) tA = false;
    else if (groupable(A, aK, aM, &lda)) tA = true;
    else {
        packA = true;
        tA = true;
        lda = std::max<int64_t>(mK, 1);
    }
    if (groupable(B, bK, bN, &ldb)) tB = false;
    else if (groupable(B, bN, bK, &ldb)) tB = true;
    else {
        packB = true;
        tB = false;
        ldb = std::max<int64_t>(mK, 1);
    }
    auto cM = dims_of(oM, info, 2), cN = dims_of(oN, info, 2);
    const int cmode = groupable(C, cM, cN, &ldc) ? 0 : groupable(C, cN, cM, &ldc) ? 1 : 2;
    // C = beta C + the column-major mM x mN product in bufC
    auto scatter_C = [&]() {
        TV t;
        t.p = bufC.d();
        t.nd = C.nd;
        int64_t st = 1;
        for (int k = 0; k < C.nd; k++) t.n[k] = C.n[k];
        for (int d : cM) {
            t.s[d] = st;
            st *= C.n[d];
        }
        for (int d : cN) {
            t.s[d] = st;
            st *= C.n[d];
        }
        permute_add(ex, 1.0, t, beta, C);
    };
    if (packA || packB) {
        SplitView va, vb;
        if (gather_view(A, aM, aK, &va) && gather_view(B, bN, bK, &vb)) {
            // the route of the product as the reordered copies would present it
            const double fl = 2.0 * double(mM) * double(mN) * double(mK);
            const Route rt = cmode == 1 ? lookup_route(ex, !tB, !tA, mN, mM, mK, fl, true)
                                        : lookup_route(ex, tA, tB, mM, mN, mK, fl, true);
            if (rt.known && rt.mixed) {
                ex.flops += fl;
                if (trace_level() >= 2)
                    std::fprintf(stderr, "ccsd_gpu gemm [%s] bf16x3 gather m %lld n %lld k %lld  %.3g flop  splits %d\n",
                                 spec, (long long)mM, (long long)mN, (long long)mK, fl, rt.splits);
                if (cmode == 0) {
                    mixed_gemm_views(ex, va, vb, mM, mN, mK, alpha, beta, C.p, ldc, rt.splits);
                } else if (cmode == 1) {
                    mixed_gemm_views(ex, vb, va, mN, mM, mK, alpha, beta, C.p, ldc, rt.splits);
                } else {
                    bufC = dalloc(mM * mN, ex.stream);
                    mixed_gemm_views(ex, va, vb, mM, mN, mK, alpha, 0.0, bufC.d(), mM, rt.splits);
                    scatter_C();
                }
                return;
            }
        }
        if (packA) Au = make_contiguous(ex, A, aK, aM, bufA);
        if (packB) Bu = make_contiguous(ex, B, bK, bN, bufB);
    }
    if (cmode == 0) {
        gemm(ex, tA, tB, mM, mN, mK, alpha, Au.p, lda, Bu.p, ldb, beta, C.p, ldc);
    } else if (cmode == 1) {
        gemm(ex, !tB, !tA, mN, mM, mK, alpha, Bu.p, ldb, Au.p, lda, beta, C.p, ldc);
    } else {
        bufC = dalloc(mM * mN, ex.stream);
        gemm(ex, tA, tB, mM, mN, mK, alpha, Au.p, lda, Bu.p, ldb, 0.0, bufC.d(), mM);
        scatter_C();
    }
}

// ---------------------------------------------------------------------------
// packing
// ---------------------------------------------------------------------------

__device__ __forceinline__ int64_t pk(int64_t x, int64_t y) {
    int64_t M = x > y ? x : y, m = x > y ? y : x;
    return M * (M + 1) / 2 + m;
}

__global__ void squareup_kernel(const double *__restrict__ packed, double *__restrict__ full, int64_t nov) {
    int64_t total = nov * nov;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = idx % nov, c = idx / nov;
        full[idx] = packed[pk(r, c)];
    }
}

void squareup(Exec &ex, const double *packed, double *full, int64_t nov) {
    squareup_kernel<<<grid_for(nov * nov, 256), 256, 0, ex.stream>>>(packed, full, nov);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

// one thread per packed element; element (M, m) with M >= m reads full(m, M) = full[m + nov*M]
__global__ void pack_half_diag_add_kernel(double alpha, const double *__restrict__ full, double *__restrict__ packed,
                                          int64_t nov) {
    int64_t total = nov * (nov + 1) / 2;
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int64_t M = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
        while (M * (M + 1) / 2 > idx) M--;
        while ((M + 1) * (M + 2) / 2 <= idx) M++;
        int64_t m = idx - M * (M + 1) / 2;
        double v = full[m + nov * M];
        if (m == M) v *= 0.5;
        packed[idx] += alpha * v;
    }
}

void pack_half_diag_add(Exec &ex, double alpha, const double *full, double *packed, int64_t nov) {
    pack_half_diag_add_kernel<<<grid_for(nov * (nov + 1) / 2, 256), 256, 0, ex.stream>>>(alpha, full, packed, nov);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------

namespace {
constexpr int RBLOCKS = 592;   // 4 x 148 SMs
constexpr int RTHREADS = 256;

__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

__device__ double block_sum(double v) {
    __shared__ double sh[32];
    v = warp_sum(v);
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (w == 0) {
        r = lane < (blockDim.x + 31) / 32 ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    __syncthreads();
    return r;
}

struct PtrList {
    const double *p[16];
};

__global__ void multi_dot_partial(const double *__restrict__ x, PtrList ys, int nys, int64_t n,
                                  double *__restrict__ partial) {
    for (int k = 0; k < nys; k++) {
        const double *y = ys.p[k];
        double acc = 0.0;
        for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
            acc += x[i] * y[i];
        acc = block_sum(acc);
        if (threadIdx.x == 0) partial[k * gridDim.x + blockIdx.x] = acc;
    }
}

__global__ void finish_partial(const double *__restrict__ partial, int nblocks, int nys, double *__restrict__ out) {
    int k = blockIdx.x;
    double acc = 0.0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) acc += partial[k * nblocks + i];
    acc = block_sum(acc);
    if (threadIdx.x == 0) out[k] = acc;
}

__global__ void fill_kernel(double *p, int64_t n, double v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

__global__ void axpby_kernel(int64_t n, double a, const double *__restrict__ x, double b, double *__restrict__ y) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        y[i] = a * x[i] + (b == 0.0 ? 0.0 : b * y[i]);
}
}  // namespace

void multi_dot(Exec &ex, const double *x, const double *const *ys, int nys, int64_t n, double *d_results) {
    if (nys == 0) return;
    REQUIRE(nys <= 16, CCSD_GPU_EINVAL, "multi_dot: at most 16 vectors");
    PtrList pl{};
    for (int k = 0; k < nys; k++) pl.p[k] = ys[k];
    DBuf part = dalloc((int64_t)RBLOCKS * nys, ex.stream);
    multi_dot_partial<<<RBLOCKS, RTHREADS, 0, ex.stream>>>(x, pl, nys, n, part.d());
    finish_partial<<<nys, RTHREADS, 0, ex.stream>>>(part.d(), RBLOCKS, nys, d_results);
    ex.launches += 2;
    CU_CHECK(cudaGetLastError());
}

void dot(Exec &ex, const double *x, const double *y, int64_t n, double *d_result) {
    const double *ys[1] = {y};
    multi_dot(ex, x, ys, 1, n, d_result);
}

void fill(Exec &ex, double *p, int64_t n, double value) {
    if (n == 0) return;
    fill_kernel<<<grid_for(n, 256), 256, 0, ex.stream>>>(p, n, value);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void axpby(Exec &ex, int64_t n, double alpha, const double *x, double beta, double *y) {
    if (n == 0) return;
    axpby_kernel<<<grid_for(n, 256), 256, 0, ex.stream>>>(n, alpha, x, beta, y);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

}  // namespace ccsd
