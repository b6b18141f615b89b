// Split-BF16 GEMM for sm_100a: D = alpha * sum_(p,q) A_p B_q^T + beta * C over bf16 planes.
//
// FP64 operands are converted once per call into NP bf16 planes (x = x_0 + x_1 [+ x_2], each plane
// the bf16 rounding of what the planes before it leave), K-major and zero padded (M to 128, N to
// 256, K to 64).  Two modes:
//   bf16x3: NP = 2, products (0,0) (0,1) (1,0), N tile 256            (~16 significant bits)
//   bf16x6: NP = 3, products (0,0) (0,1) (1,0) (0,2) (1,1) (2,0), N tile 128   (~24 bits)
// Both keep two 96 KB shared-memory stages.  The kernel is persistent and warp specialised: one
// thread issues TMA loads of the 128B-swizzled operand tiles into the ring of stages, one thread
// issues tcgen05.mma (kind::f16, FP32 accumulation in TMEM) for every product of every 16-wide K
// slice, and four warps drain the 128 x BN accumulator through tcgen05.ld and write FP64
// column-major output (alpha/beta applied in FP64).  The tensor cores' FP32
// accumulation loses a little at every MMA step, so long K ranges are cut into chunks
// (Exec::k_chunk, 4096 by default): each chunk accumulates in one TMEM buffer and the epilogue
// adds it to the FP64 output while the next chunk accumulates in the other; the same CTA takes
// the chunks of a tile in order, so the sum is deterministic.  Every mbarrier wait is bounded;
// on time-out the kernel records an error code in the caller's error word (one per context),
// skips its remaining work, waits (bounded) for the copies it has in flight and frees its TMEM.
#include <cuda.h>
#include <cuda_bf16.h>

#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <mutex>
#include <type_traits>

#include "mixed_gemm.cuh"
#include "tc_common.cuh"

namespace ccsd {

using namespace tc;

namespace {

constexpr int BM = 128;
constexpr int BK = 64;                     // K padding of the planes: one 128-byte swizzle row of bf16
constexpr int B_ROW_PAD = 256;             // B operand rows are padded to 256 in both modes
constexpr int THREADS = 192;              // producer warp, MMA warp, four epilogue warps
constexpr int EPI_THREADS = 128;
constexpr long long WAIT_CYCLES = 4000000000ll;   // ~2 s at 2 GHz: far above any legitimate wait
// error codes written to the caller's error word when a bounded wait runs out
constexpr int ERR_PRODUCER = 1, ERR_MMA_FULL = 2, ERR_EPILOGUE = 3, ERR_MMA_ACC = 4, ERR_DONE = 5, ERR_DRAIN = 6;

// plane count, N tile, K block of one pipeline stage (64 bf16 in 128-byte swizzled rows, or 32 in
// 64-byte rows) and stage count of one mode.  Four 48 KB stages of 32-wide blocks measured 5 %
// slower than two 96 KB stages of 64-wide blocks at 10240^3 and equal at 4096 x 4096 x 1200.
template <int NP_, int BN_, int KB_ = 64, int STAGES_ = 2>
struct Mode {
    static constexpr int NP = NP_;
    static constexpr int BN = BN_;
    static constexpr int KB = KB_;
    static constexpr int STAGES = STAGES_;
    static constexpr int ROW_BYTES = 2 * KB;
    static constexpr int NPROD = NP == 2 ? 3 : 6;
    static constexpr int A_TILE = BM * KB * 2;       // bytes per plane
    static constexpr int B_TILE = BN * KB * 2;
    static constexpr int STAGE_BYTES = NP * (A_TILE + B_TILE);
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/;
    static constexpr uint32_t TMEM_COLS = 2 * BN;    // two FP32 accumulators of 128 lanes x BN columns
    // kind::f16 instruction descriptor: BF16 x BF16 -> F32, both K-major, M = 128, N = BN
    static constexpr uint32_t IDESC =
        (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
    // plane pair (A plane, B plane) of product p, largest products first
    __host__ __device__ static constexpr int pa(int p) { return p == 2 || p == 4 ? 1 : (p == 5 ? 2 : 0); }
    __host__ __device__ static constexpr int pb(int p) { return p == 1 || p == 4 ? 1 : (p == 3 ? 2 : 0); }
};
using ModeX3 = Mode<2, 256>;
using ModeX6 = Mode<3, 128>;
static_assert(ModeX3::STAGE_BYTES == 96 * 1024 && ModeX6::STAGE_BYTES == 96 * 1024, "stage size");
static_assert(B_ROW_PAD % ModeX3::BN == 0 && B_ROW_PAD % ModeX6::BN == 0, "B padding");

}  // namespace

// FP64 column-major output with alpha/beta
struct EpiF64 {
    static constexpr bool kChunked = true;   // can accumulate K chunks into the output
    double *C;
    long long ldc;
    int M, N;
    double alpha, beta;
    long long zstride = 0;   // split-K: slice z writes its partial product at C + z*zstride
    long long zoff = 0;
    __device__ __forceinline__ void tile_setup(int z) { zoff = (long long)z * zstride; }
    __device__ __forceinline__ void row_setup(int) {}
    // 16 consecutive columns of one row.  first: the first K chunk of the tile (beta applies);
    // later chunks add to what is there, in FP64.  The 16 old values are loaded before any store so
    // their L2 latencies overlap.
    __device__ __forceinline__ void apply16(int row, int col0, const float (&v)[16], bool first) const {
        if (row >= M) return;
        double *base = C + zoff + (long long)col0 * ldc + row;
        const bool need_old = !first || beta != 0.0;
        double old[16];
#pragma unroll
        for (int j = 0; j < 16; j++) old[j] = (need_old && col0 + j < N) ? __ldcg(base + (long long)j * ldc) : 0.0;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            if (col0 + j < N) {
                double r = alpha * (double)v[j];
                if (!first) r += old[j];
                else if (beta != 0.0) r += beta * old[j];
                base[(long long)j * ldc] = r;
            }
        }
    }
};

// v as np bf16 planes at out[idx], out[plane + idx], ...: each plane is the bf16 rounding of what
// the planes before it leave over (the differences are exact in FP32)
__device__ __forceinline__ void store_split_planes(__nv_bfloat16 *out, size_t plane, size_t idx, float v, int np) {
    __nv_bfloat16 hi = __float2bfloat16(v);
    const float r = v - __bfloat162float(hi);
    __nv_bfloat16 mid = __float2bfloat16(r);
    out[idx] = hi;
    out[plane + idx] = mid;
    if (np == 3) out[2 * plane + idx] = __float2bfloat16(r - __bfloat162float(mid));
}

// ovvv integrals of the untransformed Cholesky vectors for the ladder's Y intermediate: row
// (c, k) = c + nv*k of L_ov, column (d, b) = d + nv*b of L_vv, so G = L_ov^T L_vv holds
// g_kcbd; written as np bf16 planes at row k + no*b, K position c + nv*d (the 32 lanes of a warp
// take consecutive c and store to consecutive addresses).
struct EpiOvvv {
    static constexpr bool kChunked = false;
    __nv_bfloat16 *out;
    size_t plane;
    long long ldk;
    int no, nv, M, N, np;
    int k, c;
    __device__ __forceinline__ void tile_setup(int) {}
    __device__ __forceinline__ void row_setup(int row) {
        k = row / nv;
        c = row - k * nv;
    }
    __device__ __forceinline__ void apply16(int row, int col0, const float (&v)[16], bool) const {
        if (row >= M) return;
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const int col = col0 + j;
            if (col >= N) return;
            const int b = col / nv, d = col - b * nv;
            const size_t idx = (size_t)(k + (long long)no * b) * ldk + c + (long long)nv * d;
            store_split_planes(out, plane, idx, v[j], np);
        }
    }
};

namespace {

// Tile t of the flattened (split, m-tile, n-tile) space.  Tiles are rasterised in groups of
// `group_m` m-tiles: inside a group the m index runs fastest, then n, so the ~148 tiles resident at
// one time cover about group_m A panels and 148/group_m B panels, which L2 serves to all of them
// (instead of every wave streaming the whole of A or B from HBM again).
struct TileMap {
    int num_mt, num_nt, nk_all, nks, group_m, bn;
    int bm = BM;            // rows of one tile (256 for a CTA pair)
    int kc;   // K blocks accumulated in TMEM before the epilogue takes the partial sum (FP64)
    int *err;               // the caller's error word (device): a bounded wait that ran out writes its code
    long long wait_cycles;  // bound of every barrier wait
    int stall_test;         // diagnostics: the producer withholds the loads of its first stage, so the
                            // MMA warp's wait for it runs out by design
    __device__ __forceinline__ void decode(int t, int &m0, int &n0, int &z, int &kt0, int &nk) const {
        const int per_split = num_mt * num_nt;
        z = t / per_split;
        const int r = t - z * per_split;
        const int per_group = group_m * num_nt;
        const int grp = r / per_group, in = r - grp * per_group;
        const int first_m = grp * group_m;
        const int gsz = min(group_m, num_mt - first_m);
        const int mt = first_m + in % gsz, nt = in / gsz;
        m0 = mt * bm;
        n0 = nt * bn;
        kt0 = z * nks;
        nk = min(nks, nk_all - kt0);
    }
};

// Persistent, warp-specialised: warp 0 = TMA producer, warp 1 = MMA issuer (and TMEM owner),
// warps 2..5 = epilogue.  Two 128 x BN FP32 accumulators in TMEM let the epilogue of one
// accumulation unit overlap the main loop of the next.
template <class MD, class Epi>
__global__ void __launch_bounds__(THREADS, 1)
split_bf16_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, TileMap map,
                   int num_tiles, Epi epi) {
    constexpr int NP = MD::NP, BN = MD::BN, A_TILE = MD::A_TILE, B_TILE = MD::B_TILE;
    constexpr int STAGE_BYTES = MD::STAGE_BYTES, STAGES = MD::STAGES, KB = MD::KB;
    constexpr uint32_t TMEM_COLS = MD::TMEM_COLS;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *acc_full = empty + STAGES;    // [2]
    uint64_t *acc_empty = acc_full + 2;     // [2]
    uint64_t *done = acc_empty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], EPI_THREADS);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // TMA producer: one ring of stages across all tiles of this CTA
            int g = 0;
            int issued[STAGES] = {};   // loads issued per stage (at most the last one is in flight)
            for (int t = blockIdx.x; t < num_tiles && !*abort_flag; t += gridDim.x) {
                int m0, n0, z, kt0, nk;
                map.decode(t, m0, n0, z, kt0, nk);
                for (int i = 0; i < nk; i++, g++) {
                    const int s = g % STAGES;
                    if (!mbar_wait(&empty[s], ((g / STAGES) & 1) ^ 1, map.wait_cycles) || *abort_flag) {
                        record_error(map.err, ERR_PRODUCER);
                        *abort_flag = 1;
                        break;
                    }
                    if (map.stall_test && g == 0) continue;   // stage 0's first phase never completes
                    issued[s]++;
                    uint8_t *st = smem + s * STAGE_BYTES;
                    mbar_expect_tx(&full[s], STAGE_BYTES);
                    const int k0 = (kt0 + i) * KB;
#pragma unroll
                    for (int p = 0; p < NP; p++) {
                        tma_load_3d(&tmA, &full[s], st + p * A_TILE, k0, m0, p);
                        tma_load_3d(&tmB, &full[s], st + NP * A_TILE + p * B_TILE, k0, n0, p);
                    }
                }
            }
            // the last load issued to each stage may still be landing (the consumers may abort
            // before they read it): wait for it, so no copy of this CTA is in flight when its
            // shared memory goes away.  In a normal run these phases complete anyway.
            for (int s = 0; s < STAGES; s++)
                if (issued[s] && !mbar_wait(&full[s], (issued[s] - 1) & 1, map.wait_cycles))
                    record_error(map.err, ERR_DRAIN);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer
            // one accumulation unit = one K chunk of one tile; units alternate between the two
            // TMEM accumulators
            int g = 0, tc = 0;
            for (int t = blockIdx.x; t < num_tiles && !*abort_flag; t += gridDim.x) {
                int m0, n0, z, kt0, nk;
                map.decode(t, m0, n0, z, kt0, nk);
                for (int c0 = 0; c0 < nk && !*abort_flag; c0 += map.kc, tc++) {
                const int acc = tc & 1;
                if (!mbar_wait(&acc_empty[acc], ((tc >> 1) & 1) ^ 1, map.wait_cycles)) {
                    record_error(map.err, ERR_MMA_ACC);
                    *abort_flag = 1;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t d = tmem + (uint32_t)(acc * BN);
                const int c1 = min(nk, c0 + map.kc);
                for (int i = c0; i < c1; i++, g++) {
                    const int s = g % STAGES;
                    if (!mbar_wait(&full[s], (g / STAGES) & 1, map.wait_cycles) || *abort_flag) {
                        record_error(map.err, ERR_MMA_FULL);
                        *abort_flag = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint8_t *st = smem + s * STAGE_BYTES;
#pragma unroll
                    for (int kk = 0; kk < KB / 16; kk++) {
                        const uint32_t ko = kk * 32;   // 16 bf16 = 32 bytes inside the swizzled row
#pragma unroll
                        for (int p = 0; p < MD::NPROD; p++) {
                            const uint8_t *ta = st + MD::pa(p) * A_TILE;
                            const uint8_t *tb = st + NP * A_TILE + MD::pb(p) * B_TILE;
                            mma_bf16(d, smem_desc_k<MD::ROW_BYTES>(ta, ko), smem_desc_k<MD::ROW_BYTES>(tb, ko), MD::IDESC,
                                     (i > c0 || kk > 0 || p > 0) ? 1u : 0u);
                        }
                    }
                    mma_commit(&empty[s]);   // frees the stage once these MMAs have read it
                }
                mma_commit(&acc_full[acc]);  // accumulator ready for the epilogue
                }
            }
            mma_commit(done);                // every MMA of this CTA has completed
        }
    } else {
        // epilogue: warp w reads TMEM lanes 32*(w % 4) .. +31
        const int quarter = warp & 3;
        int tc = 0;
        bool aborted = false;
        for (int t = blockIdx.x; t < num_tiles && !aborted; t += gridDim.x) {
            int m0, n0, z, kt0, nk;
            map.decode(t, m0, n0, z, kt0, nk);
            for (int c0 = 0; c0 < nk; c0 += map.kc, tc++) {
            const int acc = tc & 1;
            bool ok = !*abort_flag && mbar_wait(&acc_full[acc], (tc >> 1) & 1, map.wait_cycles);
            __syncwarp();
            if (!ok || *abort_flag) {
                record_error(map.err, ERR_EPILOGUE);
                *abort_flag = 1;
                aborted = true;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int row = m0 + quarter * 32 + lane;
            epi.tile_setup(z);
            epi.row_setup(row);
            const uint32_t base = tmem + (uint32_t)(acc * BN) + ((uint32_t)(quarter * 32) << 16);
#pragma unroll 1
            for (int cc = 0; cc < BN; cc += 16) {
                float v[16];
                tmem_ld16(base + (uint32_t)cc, v);
                epi.apply16(row, n0 + cc, v, c0 == 0);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&acc_empty[acc])) : "memory");
            }
        }
    }
    __syncthreads();
    // all MMAs complete before the TMEM is released
    if (!mbar_wait(done, 0, map.wait_cycles)) record_error(map.err, ERR_DONE);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}
// The same GEMM on a pair of CTAs (a cluster of two on neighbouring SMs) sharing one tcgen05 MMA of
// M = 256 (cta_group::2): each CTA stages its own 128 rows of A and half of the 256-wide B tile, so
// a CTA moves 64 KB per K block instead of 96 KB and three stages fit in its shared memory (the
// producer runs two K blocks ahead of the tensor cores instead of one).  CTA 0 of the pair issues
// the MMAs and waits for both CTAs' loads on its own barriers (the loads of CTA 1 complete on CTA 0's
// barrier); its commits arrive on the stage and accumulator barriers of both CTAs.  Each CTA's
// epilogue drains its own TMEM rows and then signals CTA 0 that the accumulator is free.
namespace {

struct PairMode {
    static constexpr int NP = 2, KB = 64, BN = 256, STAGES = 3;
    static constexpr int A_TILE = BM * KB * 2;          // 128 rows of one plane
    static constexpr int B_TILE = (BN / 2) * KB * 2;    // this CTA's half of the B tile
    static constexpr int STAGE_BYTES = NP * (A_TILE + B_TILE);
    static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
    static constexpr uint32_t TMEM_COLS = 2 * BN;
    static constexpr uint32_t IDESC =
        (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(256 >> 4) << 24);
};
static_assert(PairMode::STAGE_BYTES == 64 * 1024, "pair stage size");

__device__ __forceinline__ void mma_bf16_pair(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                              uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

template <class Epi>
__global__ void __launch_bounds__(THREADS, 1)
split_bf16_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, TileMap map,
                       int num_tiles, Epi epi) {
    using MD = PairMode;
    constexpr int A_TILE = MD::A_TILE, B_TILE = MD::B_TILE, STAGE_BYTES = MD::STAGE_BYTES, STAGES = MD::STAGES;
    constexpr int KB = MD::KB, BN = MD::BN;
    constexpr uint32_t TMEM_COLS = MD::TMEM_COLS;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *acc_full = empty + STAGES;    // [2]
    uint64_t *acc_empty = acc_full + 2;     // [2], used on CTA 0
    uint64_t *done = acc_empty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool lead = rank == 0;
    const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int a = 0; a < 2; a++) {
            mbar_init(&acc_full[a], 1);
            mbar_init(&acc_empty[a], 2 * (EPI_THREADS / 32));   // one arrival per epilogue warp of each CTA
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    cluster_sync();   // both CTAs' barriers exist before any load, commit or arrival crosses the pair
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // TMA producer of this CTA: its A rows and its half of B; CTA 0 expects both CTAs' bytes
            int g = 0;
            int issued[STAGES] = {};
            for (int t = pair; t < num_tiles && !*abort_flag; t += npairs) {
                int m0, n0, z, kt0, nk;
                map.decode(t, m0, n0, z, kt0, nk);
                for (int i = 0; i < nk; i++, g++) {
                    const int s = g % STAGES;
                    if (!mbar_wait(&empty[s], ((g / STAGES) & 1) ^ 1, map.wait_cycles) || *abort_flag) {
                        record_error(map.err, ERR_PRODUCER);
                        *abort_flag = 1;
                        break;
                    }
                    if (map.stall_test && g == 0) continue;   // stage 0's first phase never completes
                    issued[s]++;
                    uint8_t *st = smem + s * STAGE_BYTES;
                    if (lead) mbar_expect_tx(&full[s], 2 * STAGE_BYTES);
                    const int k0 = (kt0 + i) * KB;
#pragma unroll
                    for (int p = 0; p < MD::NP; p++) {
                        tma_load_3d_pair(&tmA, &full[s], st + p * A_TILE, k0, m0 + BM * (int)rank, p);
                        tma_load_3d_pair(&tmB, &full[s], st + MD::NP * A_TILE + p * B_TILE, k0, n0 + (BN / 2) * (int)rank,
                                         p);
                    }
                }
            }
            // CTA 0 waits for the last load of each stage (both CTAs' bytes land on its barrier); CTA 1
            // keeps its shared memory until the final cluster barrier, which CTA 0 reaches after this
            if (lead)
                for (int s = 0; s < STAGES; s++)
                    if (issued[s] && !mbar_wait(&full[s], (issued[s] - 1) & 1, map.wait_cycles))
                        record_error(map.err, ERR_DRAIN);
        }
    } else if (warp == 1) {
        if (lane == 0 && lead) {
            // MMA issuer of the pair
            int g = 0, tc = 0;
            for (int t = pair; t < num_tiles && !*abort_flag; t += npairs) {
                int m0, n0, z, kt0, nk;
                map.decode(t, m0, n0, z, kt0, nk);
                for (int c0 = 0; c0 < nk && !*abort_flag; c0 += map.kc, tc++) {
                    const int acc = tc & 1;
                    if (!mbar_wait(&acc_empty[acc], ((tc >> 1) & 1) ^ 1, map.wait_cycles)) {
                        record_error(map.err, ERR_MMA_ACC);
                        *abort_flag = 1;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t d = tmem + (uint32_t)(acc * BN);
                    const int c1 = min(nk, c0 + map.kc);
                    for (int i = c0; i < c1; i++, g++) {
                        const int s = g % STAGES;
                        if (!mbar_wait(&full[s], (g / STAGES) & 1, map.wait_cycles) || *abort_flag) {
                            record_error(map.err, ERR_MMA_FULL);
                            *abort_flag = 1;
                            break;
                        }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        const uint8_t *st = smem + s * STAGE_BYTES;
#pragma unroll
                        for (int kk = 0; kk < KB / 16; kk++) {
                            const uint32_t ko = kk * 32;
#pragma unroll
                            for (int p = 0; p < 3; p++) {
                                // hi*hi, hi*lo, lo*hi
                                const uint8_t *ta = st + (p == 2 ? 1 : 0) * A_TILE;
                                const uint8_t *tb = st + MD::NP * A_TILE + (p == 1 ? 1 : 0) * B_TILE;
                                mma_bf16_pair(d, smem_desc_k<128>(ta, ko), smem_desc_k<128>(tb, ko), MD::IDESC,
                                              (i > c0 || kk > 0 || p > 0) ? 1u : 0u);
                            }
                        }
                        mma_commit_pair(&empty[s]);
                    }
                    mma_commit_pair(&acc_full[acc]);
                }
            }
            mma_commit_pair(done);
        }
    } else {
        // epilogue: this CTA's 128 rows; warp w reads TMEM lanes 32*(w % 4) .. +31
        const int quarter = warp & 3;
        int tc = 0;
        bool aborted = false;
        for (int t = pair; t < num_tiles && !aborted; t += npairs) {
            int m0, n0, z, kt0, nk;
            map.decode(t, m0, n0, z, kt0, nk);
            for (int c0 = 0; c0 < nk; c0 += map.kc, tc++) {
                const int acc = tc & 1;
                bool ok = !*abort_flag && mbar_wait(&acc_full[acc], (tc >> 1) & 1, map.wait_cycles);
                __syncwarp();
                if (!ok || *abort_flag) {
                    record_error(map.err, ERR_EPILOGUE);
                    *abort_flag = 1;
                    aborted = true;
                    break;
                }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const int row = m0 + BM * (int)rank + quarter * 32 + lane;
                epi.tile_setup(z);
                epi.row_setup(row);
                const uint32_t base = tmem + (uint32_t)(acc * BN) + ((uint32_t)(quarter * 32) << 16);
#pragma unroll 1
                for (int cc = 0; cc < BN; cc += 16) {
                    float v[16];
                    tmem_ld16(base + (uint32_t)cc, v);
                    epi.apply16(row, n0 + cc, v, c0 == 0);
                }
                asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                __syncwarp();
                if (lane == 0) arrive_cta0(&acc_empty[acc]);
            }
        }
    }
    __syncthreads();
    // every MMA of the pair complete before the TMEM is released (CTA 0's commit reaches both CTAs)
    if (!mbar_wait(done, 0, map.wait_cycles)) record_error(map.err, ERR_DONE);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    cluster_sync();   // no arrival or load of either CTA is still headed for the other
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

}  // namespace

// FP64 operand (a strided gather: element (r, k) at p[roff(r) + koff(k)], the row and K indices
// each spread over up to four tensor dimensions) -> np bf16 planes, K-major [plane][Rp][Kp]: plane q
// holds the bf16 rounding of x minus the planes before it.  One pass reads the FP64 tensor in
// whatever order its dimensions lie and writes the planes, so an operand whose indices are not in
// GEMM order needs no FP64 reordering copy first.
//
// The work is cut into boxes of 32 x 32 in the digits of two tensor dimensions: `a`, the first K
// dimension (consecutive a are consecutive K positions, so the stores run along K), and `b`, the
// tensor's unit-stride dimension where that is another one (so the loads run along it; otherwise the
// first row dimension).  Every other digit is fixed per box.  Each warp takes boxes on its own: 8-byte
// asynchronous copies (cp.async) along the unit-stride digit into its shared-memory tile, then bf16
// planes stored along a.  Padding rows and K positions are cleared separately.
constexpr int GS_WARPS = 4, GS_T = 32, GS_LD = GS_T + 1, GS_REST = 6;

struct GatherPlan {
    const double *p;
    long long na, nb;           // extents of the a and b digits
    long long sa, sb;           // their memory strides
    long long orb, okb;         // output row / K step of one b (a steps K by 1)
    int lanes_on_a;             // the loads run along a (a has unit stride)
    int nrest;
    long long rn[GS_REST], rs[GS_REST], ror[GS_REST], rok[GS_REST];
};

__device__ __forceinline__ void cp_async8(double *dst, const double *src, bool valid) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src), "r"(valid ? 8 : 0) : "memory");
}

__global__ void __launch_bounds__(GS_WARPS * 32) gather_split_kernel(GatherPlan g, long long ntiles, int Rp, int Kp,
                                                                      int np, __nv_bfloat16 *__restrict__ out) {
    __shared__ __align__(16) double tiles[GS_WARPS][GS_T * GS_LD];   // element (i, j) at [j * GS_LD + i]
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *tile = tiles[warp];
    const long long ta = (g.na + GS_T - 1) / GS_T, tb = (g.nb + GS_T - 1) / GS_T;
    const size_t plane = (size_t)Rp * Kp;
    for (long long t = (long long)blockIdx.x * GS_WARPS + warp; t < ntiles; t += (long long)gridDim.x * GS_WARPS) {
        const long long ca = t % ta, t1 = t / ta, cb = t1 % tb;
        long long rest = t1 / tb, mem = 0, row = 0, kpos = 0;
        for (int d = 0; d < g.nrest; d++) {
            const long long q = rest / g.rn[d], x = rest - q * g.rn[d];
            mem += x * g.rs[d];
            row += x * g.ror[d];
            kpos += x * g.rok[d];
            rest = q;
        }
        const long long a0 = GS_T * ca, b0 = GS_T * cb;
        const int na = (int)min(g.na - a0, (long long)GS_T), nb = (int)min(g.nb - b0, (long long)GS_T);
        const double *base = g.p + mem + a0 * g.sa + b0 * g.sb;
        if (g.lanes_on_a) {
            const double *src = base + lane * g.sa;
#pragma unroll 8
            for (int j = 0; j < GS_T; j++) cp_async8(tile + j * GS_LD + lane, lane < na && j < nb ? src + j * g.sb : g.p,
                                                     lane < na && j < nb);
        } else {
            const double *src = base + lane * g.sb;
#pragma unroll 8
            for (int i = 0; i < GS_T; i++) cp_async8(tile + lane * GS_LD + i, i < na && lane < nb ? src + i * g.sa : g.p,
                                                     i < na && lane < nb);
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        __syncwarp();
        if (lane < na) {
            const long long r_base = row + b0 * g.orb, k_base = kpos + a0 + lane + b0 * g.okb;
            for (int j = 0; j < nb; j++) {
                double y = tile[j * GS_LD + lane];
                __nv_bfloat16 *o = out + (size_t)(r_base + j * g.orb) * Kp + (k_base + j * g.okb);
                for (int q = 0; q < np; q++) {
                    const __nv_bfloat16 h = __double2bfloat16(y);
                    o[q * plane] = h;
                    y -= (double)__bfloat162float(h);
                }
            }
        }
        __syncwarp();
    }
}

// C = beta C + sum_z P_z  (P_z dense m x n, z-major)
__global__ void sum_splits_kernel(const double *__restrict__ P, int splits, int64_t m, int64_t n, double beta,
                                  double *__restrict__ C, int64_t ldc) {
    for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < m * n;
         idx += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = idx % m, c = idx / m;
        double acc = 0.0;
        for (int z = 0; z < splits; z++) acc += P[(int64_t)z * m * n + idx];
        double *dst = C + r + ldc * c;
        *dst = beta != 0.0 ? beta * *dst + acc : acc;
    }
}

// planes x rows x K tensor of bf16, box (kb, box_rows, 1) with the swizzle of kb-wide rows; rows
// beyond `rows` read as zero
CUtensorMap make_map(void *base, int64_t rows, int64_t Kp, int box_rows, int64_t plane_stride, int planes,
                     int kb = BK) {
    CUtensorMap m;
    REQUIRE((reinterpret_cast<uintptr_t>(base) & 15) == 0, CCSD_GPU_EINVAL, "tensor map base must be 16-byte aligned");
    cuuint64_t dims[3] = {(cuuint64_t)Kp, (cuuint64_t)rows, (cuuint64_t)planes};
    cuuint64_t strides[2] = {(cuuint64_t)Kp * 2, (cuuint64_t)plane_stride * 2};
    cuuint32_t box[3] = {(cuuint32_t)kb, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, base, dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE,
                             kb == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    REQUIRE(r == CUDA_SUCCESS, CCSD_GPU_ECUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return m;
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

int sm_count() {
    static std::atomic<int> nsm[128] = {};   // contexts on several host threads share it
    int dev = 0;
    CU_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 128) dev = 0;
    int v = nsm[dev].load(std::memory_order_relaxed);
    if (!v) {
        CU_CHECK(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
        nsm[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

// A: a_rows rows of NP planes with stride a_plane; B likewise; the grid covers m_out x n_out output
// elements (rounded up to the tile); mnk = m * n * k of the product for the FLOP count.
template <class MD, class Epi>
void launch_mode(Exec &ex, const __nv_bfloat16 *A, int64_t a_rows, int64_t a_plane, int64_t m_out,
                 const __nv_bfloat16 *B, int64_t b_rows, int64_t b_plane, int64_t n_out, int64_t Kp, const Epi &epi,
                 double mnk, int splits) {
    const int64_t Mp = round_up(m_out, BM), Np = round_up(n_out, MD::BN);
    REQUIRE(Kp % BK == 0 && Kp > 0 && Mp > 0 && Np > 0, CCSD_GPU_EINVAL, "tc gemm: bad padding");
    CU_CHECK(cudaFuncSetAttribute(split_bf16_gemm_kernel<MD, Epi>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  MD::SMEM_BYTES));
    CUtensorMap ta = make_map(const_cast<__nv_bfloat16 *>(A), a_rows, Kp, BM, a_plane, MD::NP, MD::KB);
    CUtensorMap tb = make_map(const_cast<__nv_bfloat16 *>(B), b_rows, Kp, MD::BN, b_plane, MD::NP, MD::KB);
    TileMap map;
    map.num_mt = (int)(Mp / BM);
    map.num_nt = (int)(Np / MD::BN);
    map.nk_all = (int)(Kp / MD::KB);
    map.nks = (map.nk_all + splits - 1) / splits;
    map.bn = MD::BN;
    map.group_m = std::min(map.num_mt, 16);
    map.kc = (Epi::kChunked && ex.k_chunk > 0) ? (int)std::max<int64_t>(1, ex.k_chunk / MD::KB) : map.nks;
    REQUIRE(ex.gemm_err != nullptr, CCSD_GPU_EINVAL, "tc gemm: no error word");
    map.err = ex.gemm_err;
    map.wait_cycles = ex.wait_cycles > 0 ? ex.wait_cycles : WAIT_CYCLES;
    map.stall_test = ex.stall_test;
    const int num_tiles = map.num_mt * map.num_nt * splits;
    dim3 grid((unsigned)std::min(num_tiles, sm_count()));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ex.prof && ex.prof->on) {
        CU_CHECK(cudaEventCreate(&e0));
        CU_CHECK(cudaEventCreate(&e1));
        CU_CHECK(cudaEventRecord(e0, ex.stream));
    }
    split_bf16_gemm_kernel<MD, Epi><<<grid, THREADS, MD::SMEM_BYTES, ex.stream>>>(ta, tb, map, num_tiles, epi);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
    if (e0) {
        CU_CHECK(cudaEventRecord(e1, ex.stream));
        ex.prof->events.emplace_back(e0, e1);
        ex.prof->flops.push_back(2.0 * MD::NPROD * mnk);
    }
}

// the two-plane GEMM on CTA pairs: tiles of 256 x 256, persistent over the pairs that can be resident
template <class Epi>
void launch_pair(Exec &ex, const __nv_bfloat16 *A, int64_t a_rows, int64_t a_plane, int64_t m_out,
                 const __nv_bfloat16 *B, int64_t b_rows, int64_t b_plane, int64_t n_out, int64_t Kp, const Epi &epi,
                 double mnk, int splits) {
    using MD = PairMode;
    const int64_t Mp = round_up(m_out, 2 * BM), Np = round_up(n_out, MD::BN);
    REQUIRE(Kp % BK == 0 && Kp > 0 && Mp > 0 && Np > 0, CCSD_GPU_EINVAL, "tc gemm: bad padding");
    auto kernel = split_bf16_pair_kernel<Epi>;
    CU_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MD::SMEM_BYTES));
    // rows beyond a buffer's own rows (the second CTA of the last pair tile) read as zero
    CUtensorMap ta = make_map(const_cast<__nv_bfloat16 *>(A), a_rows, Kp, BM, a_plane, MD::NP, MD::KB);
    CUtensorMap tb = make_map(const_cast<__nv_bfloat16 *>(B), b_rows, Kp, MD::BN / 2, b_plane, MD::NP, MD::KB);
    TileMap map;
    map.bm = 2 * BM;
    map.num_mt = (int)(Mp / (2 * BM));
    map.num_nt = (int)(Np / MD::BN);
    map.nk_all = (int)(Kp / MD::KB);
    map.nks = (map.nk_all + splits - 1) / splits;
    map.bn = MD::BN;
    map.group_m = std::min(map.num_mt, 8);
    map.kc = (Epi::kChunked && ex.k_chunk > 0) ? (int)std::max<int64_t>(1, ex.k_chunk / MD::KB) : map.nks;
    REQUIRE(ex.gemm_err != nullptr, CCSD_GPU_EINVAL, "tc gemm: no error word");
    map.err = ex.gemm_err;
    map.wait_cycles = ex.wait_cycles > 0 ? ex.wait_cycles : WAIT_CYCLES;
    map.stall_test = ex.stall_test;
    const int num_tiles = map.num_mt * map.num_nt * splits;
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = MD::SMEM_BYTES;
    cfg.stream = ex.stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    static int max_pairs[128] = {};
    int dev = 0;
    CU_CHECK(cudaGetDevice(&dev));
    int &mp = max_pairs[dev & 127];
    if (mp == 0) {
        cfg.gridDim = dim3((unsigned)(2 * (sm_count() / 2)));
        int n = 0;
        CU_CHECK(cudaOccupancyMaxActiveClusters(&n, kernel, &cfg));
        mp = std::max(1, n);
    }
    cfg.gridDim = dim3((unsigned)(2 * std::min(num_tiles, mp)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (ex.prof && ex.prof->on) {
        CU_CHECK(cudaEventCreate(&e0));
        CU_CHECK(cudaEventCreate(&e1));
        CU_CHECK(cudaEventRecord(e0, ex.stream));
    }
    CU_CHECK(cudaLaunchKernelEx(&cfg, kernel, ta, tb, map, num_tiles, epi));
    ex.launches++;
    if (e0) {
        CU_CHECK(cudaEventRecord(e1, ex.stream));
        ex.prof->events.emplace_back(e0, e1);
        ex.prof->flops.push_back(2.0 * 3 * mnk);
    }
}

// CTA pairs for two-plane FP64-output products with at least one full pair tile of rows, when
// CCSD_GPU_PAIR_GEMM=1.  Off by default: at 10240^3 the pair runs at the single-CTA kernel's speed
// (4.77 vs 4.75 ms, both near the power-capped bf16 rate), and the 256-row tiles pad the ladder's
// 528-row operand further than 128-row tiles do.
bool pair_gemm_on() {
    static const bool on = [] {
        const char *e = std::getenv("CCSD_GPU_PAIR_GEMM");
        return e && e[0] == '1';
    }();
    return on;
}

// pair: the CTA-pair kernel for this launch (a route the autotuner measured), else the default
template <class Epi>
void launch_tc(Exec &ex, int planes, const __nv_bfloat16 *A, int64_t a_rows, int64_t a_plane, int64_t m_out,
               const __nv_bfloat16 *B, int64_t b_rows, int64_t b_plane, int64_t n_out, int64_t Kp, const Epi &epi,
               double mnk, int splits = 1, bool pair = false) {
    if constexpr (std::is_same<Epi, EpiF64>::value) {
        if (planes == 2 && m_out >= 2 * BM && (pair || pair_gemm_on())) {
            launch_pair(ex, A, a_rows, a_plane, m_out, B, b_rows, b_plane, n_out, Kp, epi, mnk, splits);
            return;
        }
    }
    if (planes == 3)
        launch_mode<ModeX6>(ex, A, a_rows, a_plane, m_out, B, b_rows, b_plane, n_out, Kp, epi, mnk, splits);
    else
        launch_mode<ModeX3>(ex, A, a_rows, a_plane, m_out, B, b_rows, b_plane, n_out, Kp, epi, mnk, splits);
}

int n_tile(int planes) { return planes == 3 ? ModeX6::BN : ModeX3::BN; }

void split_view(Exec &ex, const SplitView &v, int64_t R, int64_t K, int64_t Rp, int64_t Kp, int planes,
                __nv_bfloat16 *out) {
    REQUIRE(R >= 1 && K >= 1 && R <= Rp && K <= Kp && Kp < (1ll << 31) && Rp < (1ll << 31), CCSD_GPU_EINVAL,
            "operand split: bad padding");
    REQUIRE(v.nr >= 1 && v.nr <= 4 && v.nk >= 1 && v.nk <= 4, CCSD_GPU_EINVAL, "operand split: 1 to 4 dims per group");
    // the digits: extent, memory stride, output row step, output K step
    struct Digit {
        long long n, s, orow, ok;
    };
    std::vector<Digit> dig;
    long long step = 1, prod_r = 1, prod_k = 1;
    for (int d = 0; d < v.nr; d++) {
        REQUIRE(v.rn[d] >= 1, CCSD_GPU_EINVAL, "operand split: bad extent");
        dig.push_back({v.rn[d], v.rs[d], step, 0});
        step *= v.rn[d];
    }
    prod_r = step;
    const int k_first = (int)dig.size();
    step = 1;
    for (int d = 0; d < v.nk; d++) {
        REQUIRE(v.kn[d] >= 1, CCSD_GPU_EINVAL, "operand split: bad extent");
        dig.push_back({v.kn[d], v.ks[d], 0, step});
        step *= v.kn[d];
    }
    prod_k = step;
    REQUIRE(prod_r == R && prod_k == K, CCSD_GPU_EINVAL, "operand split: view extents do not match the operand");
    // a: the first K digit; b: the unit-stride digit if another one has it, else the first row digit
    const int ia = k_first;
    int ib = -1;
    for (int d = 0; d < (int)dig.size(); d++)
        if (d != ia && dig[d].n > 1 && dig[d].s == 1 && dig[ia].s != 1) ib = d;
    if (ib < 0) {
        for (int d = 0; d < (int)dig.size(); d++)
            if (d != ia && dig[d].n > 1) {
                ib = d;
                break;
            }
    }
    GatherPlan g{};
    g.p = v.p;
    g.na = dig[ia].n;
    g.sa = dig[ia].s;
    g.lanes_on_a = dig[ia].s == 1 || ib < 0 || dig[ib].s != 1;
    if (ib >= 0) {
        g.nb = dig[ib].n;
        g.sb = dig[ib].s;
        g.orb = dig[ib].orow;
        g.okb = dig[ib].ok;
    } else {
        g.nb = 1;
    }
    for (int d = 0; d < (int)dig.size(); d++) {
        if (d == ia || d == ib || dig[d].n == 1) continue;
        REQUIRE(g.nrest < GS_REST, CCSD_GPU_EINVAL, "operand split: too many dims");
        g.rn[g.nrest] = dig[d].n;
        g.rs[g.nrest] = dig[d].s;
        g.ror[g.nrest] = dig[d].orow;
        g.rok[g.nrest] = dig[d].ok;
        g.nrest++;
    }
    const long long ntiles = ((g.na + GS_T - 1) / GS_T) * ((g.nb + GS_T - 1) / GS_T) * (R * K / (g.na * g.nb));
    // padding: the K positions [K, Kp) of every row of every plane, and the rows [R, Rp)
    const size_t eb = sizeof(__nv_bfloat16);
    if (Kp > K)
        CU_CHECK(cudaMemset2DAsync(out + K, Kp * eb, 0, (Kp - K) * eb, (size_t)planes * Rp, ex.stream));
    if (Rp > R)
        CU_CHECK(cudaMemset2DAsync(out + R * Kp, Rp * Kp * eb, 0, (Rp - R) * Kp * eb, planes, ex.stream));
    const int blocks = (int)std::min<long long>((ntiles + GS_WARPS - 1) / GS_WARPS, (long long)sm_count() * 6);
    gather_split_kernel<<<blocks, GS_WARPS * 32, 0, ex.stream>>>(g, ntiles, (int)Rp, (int)Kp, planes, out);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void split(Exec &ex, const double *src, int64_t sr, int64_t sk, int64_t R, int64_t K, int64_t Rp, int64_t Kp,
           int planes, __nv_bfloat16 *out) {
    split_view(ex, matrix_view(src, R, sr, K, sk), R, K, Rp, Kp, planes, out);
}

int check_planes(int planes) {
    REQUIRE(planes == 2 || planes == 3, CCSD_GPU_EINVAL, "split-bf16 planes must be 2 or 3");
    return planes;
}

// K splits for an output of `tiles` tiles over nkt K blocks: the count (up to 4, at least 16 K
// blocks per split) that fills the last wave of the persistent grid best; a split must gain at
// least 10 % of wave efficiency to pay for its partial-sum pass.
int wave_splits(int64_t tiles, int64_t nkt) {
    const int64_t nsm = sm_count();
    auto eff = [&](int64_t s) {
        const int64_t units = tiles * s;
        return double(units) / double((units + nsm - 1) / nsm * nsm);
    };
    int best = 1;
    double best_eff = eff(1);
    for (int s = 2; s <= 4; s++) {
        if (nkt / s < 16) break;
        if (eff(s) > best_eff * 1.10) {
            best = s;
            best_eff = eff(s);
        }
    }
    return best;
}

}  // namespace

int tc_default_splits(int64_t m, int64_t n, int64_t k, int planes) {
    // split K when the output tiles cannot fill the SMs: deterministic partial products, then a sum
    const int64_t tiles = (round_up(m, BM) / BM) * (round_up(n, n_tile(planes)) / n_tile(planes));
    const int64_t nkt = round_up(k, BK) / BK, nsm = sm_count();
    if (!(tiles < nsm && nkt >= 16)) return 1;
    const int64_t want = std::min<int64_t>((2 * nsm + tiles - 1) / tiles, nkt / 8);
    const int64_t per = (nkt + want - 1) / want;
    return (int)((nkt + per - 1) / per);
}

std::vector<int> tc_split_candidates(int64_t m, int64_t n, int64_t k, int planes) {
    const int64_t tiles = (round_up(m, BM) / BM) * (round_up(n, n_tile(planes)) / n_tile(planes));
    const int64_t nkt = round_up(k, BK) / BK, nsm = sm_count();
    std::vector<int> out{1};
    auto add = [&](int64_t s, int64_t min_blocks) {
        if (s < 2 || s > 64 || nkt / s < min_blocks) return;
        if (std::find(out.begin(), out.end(), (int)s) == out.end()) out.push_back((int)s);
    };
    add(tc_default_splits(m, n, k, planes), 1);
    if (tiles >= nsm) {
        for (int s = 2; s <= 4; s++) add(s, 16);
    } else {
        // counts whose units fill about j waves of the persistent grid
        for (int j = 1; j <= 4; j++) add(j * nsm / tiles, 4);
    }
    // the same K splits on CTA pairs (256 x 256 tiles) for products with a full pair tile of rows
    if (planes == 2 && m >= 2 * BM) {
        const size_t single = out.size();
        for (size_t i = 0; i < single; i++) out.push_back(PAIR_ROUTE + out[i]);
    }
    return out;
}

void mixed_gemm_views(Exec &ex, const SplitView &A, const SplitView &B, int64_t m, int64_t n, int64_t k, double alpha,
                      double beta, double *C, int64_t ldc, int splits) {
    REQUIRE(m < (1ll << 31) && n < (1ll << 31) && k < (1ll << 31), CCSD_GPU_EINVAL, "mixed_gemm: size too large");
    const int np = check_planes(ex.planes);
    const int64_t Kp = round_up(k, BK), Mp = round_up(m, BM), Np = round_up(n, B_ROW_PAD);
    DBuf a(sizeof(__nv_bfloat16) * np * Mp * Kp, ex.stream), b(sizeof(__nv_bfloat16) * np * Np * Kp, ex.stream);
    split_view(ex, A, m, k, Mp, Kp, np, a.as<__nv_bfloat16>());
    split_view(ex, B, n, k, Np, Kp, np, b.as<__nv_bfloat16>());
    const bool pair = splits >= PAIR_ROUTE;
    if (pair) splits -= PAIR_ROUTE;
    if (splits <= 0) splits = tc_default_splits(m, n, k, np);
    splits = std::max(1, std::min<int>(splits, (int)(Kp / BK)));
    const double mnk = double(m) * double(n) * double(k);
    if (splits <= 1) {
        EpiF64 epi{C, (long long)ldc, (int)m, (int)n, alpha, beta};
        launch_tc(ex, np, a.as<__nv_bfloat16>(), Mp, Mp * Kp, m, b.as<__nv_bfloat16>(), Np, Np * Kp, n, Kp, epi, mnk, 1,
                  pair);
        return;
    }
    DBuf part = dalloc((int64_t)splits * m * n, ex.stream);
    EpiF64 epi{part.d(), (long long)m, (int)m, (int)n, alpha, 0.0, (long long)m * n};
    launch_tc(ex, np, a.as<__nv_bfloat16>(), Mp, Mp * Kp, m, b.as<__nv_bfloat16>(), Np, Np * Kp, n, Kp, epi, mnk,
              splits, pair);
    sum_splits_kernel<<<(unsigned)std::min<int64_t>((m * n + 255) / 256, 148 * 64), 256, 0, ex.stream>>>(
        part.d(), splits, m, n, beta, C, ldc);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

SplitView matrix_view(const double *p, int64_t rows, int64_t sr, int64_t K, int64_t sk) {
    SplitView v{};
    v.p = p;
    v.nr = v.nk = 1;
    v.rn[0] = std::max<int64_t>(rows, 1);
    v.rs[0] = sr;
    v.kn[0] = std::max<int64_t>(K, 1);
    v.ks[0] = sk;
    return v;
}

void mixed_gemm(Exec &ex, bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha, const double *A,
                int64_t lda, const double *B, int64_t ldb, double beta, double *C, int64_t ldc, int splits) {
    // op(A)(r, kk): A[r + lda kk] (N) or A[kk + lda r] (T); B operand rows are output columns:
    // op(B)(kk, c) = B[kk + ldb c] (N) or B[c + ldb kk] (T)
    const SplitView a = transA ? matrix_view(A, m, lda, k, 1) : matrix_view(A, m, 1, k, lda);
    const SplitView b = transB ? matrix_view(B, n, 1, k, ldb) : matrix_view(B, n, ldb, k, 1);
    mixed_gemm_views(ex, a, b, m, n, k, alpha, beta, C, ldc, splits);
}

int64_t tc_pad_rows_a(int64_t m) { return round_up(m, BM); }
int64_t tc_pad_rows_b(int64_t n) { return round_up(n, B_ROW_PAD); }
int64_t tc_pad_k(int64_t k) { return round_up(k, BK); }

void split_rows(Exec &ex, const double *src, int64_t sr, int64_t sk, int64_t R, int64_t K, int64_t Rp, int64_t Kp,
                __nv_bfloat16 *out) {
    REQUIRE(Rp % 32 == 0 && Kp % 32 == 0, CCSD_GPU_EINVAL, "split_rows: padding must be a multiple of 32");
    split(ex, src, sr, sk, R, K, Rp, Kp, check_planes(ex.planes), out);
}

void tc_gemm_f64(Exec &ex, const __nv_bfloat16 *A, int64_t Mp, const __nv_bfloat16 *B, int64_t Np, int64_t Kp,
                 int64_t m, int64_t n, int64_t k_true, double alpha, double beta, double *C, int64_t ldc,
                 int splits) {
    REQUIRE(Mp >= round_up(m, BM) && Np >= round_up(n, B_ROW_PAD), CCSD_GPU_EINVAL, "tc_gemm_f64: bad padding");
    const int np = check_planes(ex.planes);
    const double mnk = double(m) * double(n) * double(k_true);
    const bool pair = splits >= PAIR_ROUTE;
    if (pair) splits -= PAIR_ROUTE;
    if (splits <= 0) splits = wave_splits(Mp / BM * (round_up(n, n_tile(np)) / n_tile(np)), Kp / BK);
    splits = std::max(1, std::min<int>(splits, (int)(Kp / BK)));
    if (splits == 1) {
        EpiF64 epi{C, (long long)ldc, (int)m, (int)n, alpha, beta};
        launch_tc(ex, np, A, Mp, Mp * Kp, m, B, Np, Np * Kp, n, Kp, epi, mnk, 1, pair);
        return;
    }
    DBuf part = dalloc((int64_t)splits * m * n, ex.stream);
    EpiF64 epi{part.d(), (long long)m, (int)m, (int)n, alpha, 0.0, (long long)m * n};
    launch_tc(ex, np, A, Mp, Mp * Kp, m, B, Np, Np * Kp, n, Kp, epi, mnk, splits, pair);
    sum_splits_kernel<<<(unsigned)std::min<int64_t>((m * n + 255) / 256, 148 * 64), 256, 0, ex.stream>>>(
        part.d(), splits, m, n, beta, C, ldc);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

void tc_gemm_ovvv(Exec &ex, const __nv_bfloat16 *Lov, int64_t ov_rows, const __nv_bfloat16 *Lvv, int64_t vv_rows,
                  int64_t Kp, int64_t no, int64_t nv, __nv_bfloat16 *out, int64_t out_rows_pad, int64_t out_ld,
                  int64_t k_true) {
    REQUIRE(out_rows_pad >= no * nv && out_ld >= nv * nv && ov_rows >= no * nv && vv_rows >= nv * nv,
            CCSD_GPU_EINVAL, "tc_gemm_ovvv: bad padding");
    EpiOvvv epi{};
    epi.out = out;
    epi.plane = (size_t)out_rows_pad * (size_t)out_ld;
    epi.ldk = out_ld;
    epi.no = (int)no;
    epi.nv = (int)nv;
    epi.M = (int)(no * nv);
    epi.N = (int)(nv * nv);
    epi.np = check_planes(ex.planes);
    launch_tc(ex, epi.np, Lov, ov_rows, ov_rows * Kp, epi.M, Lvv, vv_rows, vv_rows * Kp, epi.N, Kp, epi,
              double(epi.M) * double(epi.N) * double(k_true));
}

int gemm_error(Exec &ex, bool reset) {
    if (!ex.gemm_err) return 0;
    int v = 0;
    CU_CHECK(cudaMemcpyAsync(&v, ex.gemm_err, sizeof(int), cudaMemcpyDeviceToHost, ex.stream));
    CU_CHECK(cudaStreamSynchronize(ex.stream));
    if (reset && v) CU_CHECK(cudaMemsetAsync(ex.gemm_err, 0, sizeof(int), ex.stream));
    return v;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the split-BF16 GEMM.
//
// Some callers cannot allocate device memory when they call in: a host program that has handed the
// whole GPU to its own memory pool up front (a Fortran driver that reserved HBM for its arrays, a
// framework whose caching allocator owns the device), or a code path that must not trigger the
// device-wide synchronisation a cudaMalloc/cudaFree can cause.  For them the operand split planes
// live in a fixed file-scope device array instead of stream-ordered allocations.
// ---------------------------------------------------------------------------

// bf16 elements of the fixed split scratch: hi and lo planes of A (Mp x Kp) and of B (Np x Kp)
constexpr int64_t NOALLOC_SCRATCH_ELEMS = 8ll << 20;   // 16 MiB, held by every GPU that loads the library
static __device__ __align__(256) __nv_bfloat16 g_noalloc_split[NOALLOC_SCRATCH_ELEMS];
// error word of the allocation-free entry point (shared by all its callers, like the scratch)
static __device__ int g_noalloc_error = 0;

namespace {
std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[128] = {};   // device address of g_noalloc_split, per device ordinal
void *g_noalloc_err[128] = {};   // device address of g_noalloc_error, per device ordinal
}  // namespace

// Device addresses of the scratch and of the error word for the current device (looked up once
// per device; the first call on a device does this set-up).
static __nv_bfloat16 *noalloc_scratch(int **err) {
    int dev = 0;
    CU_CHECK(cudaGetDevice(&dev));
    REQUIRE(dev >= 0 && dev < 128, CCSD_GPU_EINVAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr, *e = nullptr;
        cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_split);
        REQUIRE(rc == cudaSuccess && p != nullptr, CCSD_GPU_ECUDA,
                std::string("cudaGetSymbolAddress of the no-alloc scratch failed: ") + cudaGetErrorString(rc));
        rc = cudaGetSymbolAddress(&e, g_noalloc_error);
        REQUIRE(rc == cudaSuccess && e != nullptr, CCSD_GPU_ECUDA,
                std::string("cudaGetSymbolAddress of the no-alloc error word failed: ") + cudaGetErrorString(rc));
        g_noalloc_err[dev] = e;
        g_noalloc_ptr[dev] = p;
    }
    *err = static_cast<int *>(g_noalloc_err[dev]);
    return static_cast<__nv_bfloat16 *>(g_noalloc_ptr[dev]);
}

void mixed_gemm_noalloc(bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha, const double *A,
                        int64_t lda, const double *B, int64_t ldb, double beta, double *C, int64_t ldc,
                        cudaStream_t stream) {
    REQUIRE(m > 0 && n > 0 && k > 0 && A && B && C, CCSD_GPU_EINVAL, "bad gemm arguments");
    REQUIRE(m < (1ll << 31) && n < (1ll << 31) && k < (1ll << 31), CCSD_GPU_EINVAL, "no-alloc GEMM: size too large");
    REQUIRE(lda >= (transA ? k : m) && ldb >= (transB ? n : k) && ldc >= m, CCSD_GPU_EINVAL, "bad leading dimension");
    const int64_t Kp = round_up(k, BK), Mp = round_up(m, BM), Np = round_up(n, B_ROW_PAD);
    const int64_t need = 2 * (Mp + Np) * Kp;
    REQUIRE(need <= NOALLOC_SCRATCH_ELEMS, CCSD_GPU_EINVAL,
            "no-alloc GEMM: 2 x (round_up(m,128) + round_up(n,256)) x round_up(k,64) = " + std::to_string(need) +
                " bf16 elements exceeds the fixed scratch of " + std::to_string(NOALLOC_SCRATCH_ELEMS));
    int *err = nullptr;
    __nv_bfloat16 *scratch = noalloc_scratch(&err);
    Exec ex;
    ex.stream = stream;
    ex.gemm_err = err;
    __nv_bfloat16 *a = scratch, *b = scratch + 2 * Mp * Kp;
    if (!transA) split(ex, A, 1, lda, m, k, Mp, Kp, 2, a);
    else split(ex, A, lda, 1, m, k, Mp, Kp, 2, a);
    if (!transB) split(ex, B, ldb, 1, n, k, Np, Kp, 2, b);
    else split(ex, B, 1, ldb, n, k, Np, Kp, 2, b);
    EpiF64 epi{C, (long long)ldc, (int)m, (int)n, alpha, beta};
    launch_tc(ex, 2, a, Mp, Mp * Kp, m, b, Np, Np * Kp, n, Kp, epi, double(m) * double(n) * double(k));
    // synchronous: the caller learns of a bounded wait that ran out from the return status
    const int code = gemm_error(ex, true);
    REQUIRE(code == 0, CCSD_GPU_ETIMEOUT, "tensor-core GEMM barrier wait timed out (code " + std::to_string(code) + ")");
}

}  // namespace ccsd
