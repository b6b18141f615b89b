// FP64-accurate GEMM on the int8 tensor cores of sm_100a (Ozaki's error-free slicing).
//
// Every row r of op(A) is scaled by 2^-ea_r (ea_r: the exponent of the power of two just above
// max_k |A_rk|) and cut into S digits of 7 bits,
//     A_rk = 2^ea_r sum_t DA_t[r,k] 2^(-7(t+1)),   DA_t integers in [-127, 127],
// exactly up to the truncation of the last digit (relative 2^-7S); the columns of op(B) the same
// with eb_c.  Then
//     C_rc = 2^(ea_r + eb_c) sum_{t,u} 2^(-7(t+u+2)) sum_k DA_t[r,k] DB_u[k,c],
// and every digit product sum_k is exact in int32: |d d'| <= 127^2, and an accumulator takes at
// most 7 products (one diagonal d = t + u) over a K chunk of at most 16384, 7 * 16384 * 127^2 < 2^31.
// Products with t + u <= S - 1 are kept; the dropped ones lie below the last digit of either
// operand.  With S = 7 the 28 products reproduce an FP64 GEMM to ~1e-14 of the largest output.
//
// Kernel: persistent, warp specialised like the split-BF16 GEMM (warp 0 issues TMA loads, warp 1
// issues tcgen05.mma.kind::i8 with int32 accumulation in TMEM, warps 2-5 drain), 128 x 128 output
// tiles, K blocks of 64 int8 (64-byte swizzled rows).  A stage holds the digit tiles of both
// operands for one K block (up to 7 + 7 tiles of 8 KB), two stages.  The diagonals of a tile are
// accumulated in passes of at most four (4 x 128 TMEM columns = all 512): pass 0 takes d = 0..3
// (digits 0..3 of both operands), pass 1 takes d = 4..S-1 (all digits).  The epilogue adds
// 2^(-7(d+2)) acc_d in FP64, scales by alpha 2^(ea_r + eb_c) and accumulates into the FP64 output;
// one CTA takes all units (K chunk, pass) of a tile in order, so the sum is deterministic.  Every
// mbarrier wait is bounded and reports to the caller's error word, as in the split-BF16 GEMM.
#include <cuda.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "ozaki_gemm.cuh"
#include "tc_common.cuh"

namespace ccsd {

using namespace tc;

namespace {

constexpr int OBM = 128, OBN = 128, OBK = 64;            // tile; K block = one 64-byte row of int8
constexpr int SLOTS = 7;                                 // digit tiles per operand in a stage
constexpr int OSTAGES = 2;
constexpr int OTHREADS = 192, OEPI = 128;
constexpr int A_TILE = OBM * OBK, B_TILE = OBN * OBK;    // bytes
constexpr int OSTAGE_BYTES = SLOTS * (A_TILE + B_TILE);
constexpr int OSMEM = OSTAGES * OSTAGE_BYTES + 1024 + 256;
constexpr uint32_t OTMEM_COLS = 512;                     // four 128-column int32 accumulators
constexpr int MAX_DIAG_PER_PASS = 4;
constexpr int OK_CHUNK = 16384;                          // K elements per exact int32 accumulation
constexpr long long OWAIT_CYCLES = 4000000000ll;
// kind::i8 instruction descriptor: S8 x S8 -> S32, both K-major, M = 128, N = 128
constexpr uint32_t IDESC_I8 = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OBN >> 3) << 17) |
                              ((uint32_t)(OBM >> 4) << 24);
static_assert(OSMEM <= 232448, "shared memory of the Ozaki GEMM");
static_assert(7 * OK_CHUNK * 127 * 127 < 2147483647ll, "int32 accumulation must stay exact");
constexpr int ERR_PRODUCER = 1, ERR_MMA_FULL = 2, ERR_EPILOGUE = 3, ERR_MMA_ACC = 4, ERR_DONE = 5, ERR_DRAIN = 6;

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(IDESC_I8), "r"(accumulate));
}

struct OzMap {
    int num_mt, num_nt, group_m;
    int nk_all;          // K blocks of 64
    int kc;              // K blocks per chunk
    int nchunks;
    int digits;          // S
    int npass;           // 1 (S <= 4) or 2
    int M, N;
    long long ldc;
    double alpha, beta;
    double *C;
    const int *ea, *eb;  // row exponents of op(A), column exponents of op(B)
    int *err;
    long long wait_cycles;
    int bm = OBM;        // rows of one tile (256 for a CTA pair)
    __device__ __forceinline__ void tile(int t, int &m0, int &n0) const {
        const int per_group = group_m * num_nt;
        const int grp = t / per_group, in = t - grp * per_group;
        const int first_m = grp * group_m;
        const int gsz = min(group_m, num_mt - first_m);
        m0 = (first_m + in % gsz) * bm;
        n0 = (in / gsz) * OBN;
    }
    // diagonals [d0, d1) of pass p and the digits they need
    __device__ __forceinline__ void pass(int p, int &d0, int &d1, int &nd) const {
        d0 = p == 0 ? 0 : MAX_DIAG_PER_PASS;
        d1 = p == 0 ? min(digits, MAX_DIAG_PER_PASS) : digits;
        nd = min(d1, digits);   // digits 0..nd-1 of both operands (t, u <= d1 - 1)
    }
};

// The MMAs of one K block for the diagonals [D0, D1) of S-digit operands, fully unrolled: the
// descriptors of digit q sit a constant offset from those of digit 0 (a 16-byte unit in the start
// field per 16 bytes, tiles of A_TILE / B_TILE bytes), so issuing an MMA costs a few integer adds.  An
// int8 MMA of 128 x 128 x 32 lasts ~64 tensor cycles; rebuilding descriptors per MMA had the single
// issuing thread, not the tensor pipe, set the pace.
// CTA-pair form of the int8 MMA (cta_group::2, M = 256 over the pair, N = 128): issued by CTA 0,
// A rows from each CTA's own shared memory, the two 64-row halves of B from the two CTAs
constexpr uint32_t IDESC_I8_PAIR = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(OBN >> 3) << 17) |
                                   ((uint32_t)(256 >> 4) << 24);

template <bool PAIR>
__device__ __forceinline__ void mma_i8_any(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    if constexpr (PAIR) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(IDESC_I8_PAIR), "r"(accumulate));
    } else {
        mma_i8(d_tmem, adesc, bdesc, accumulate);
    }
}

template <int S, int D0, int D1, bool PAIR, int BT>
__device__ __forceinline__ void issue_kblock(uint32_t tmem, uint64_t a0, uint64_t b0, bool first_kb) {
#pragma unroll
    for (int kk = 0; kk < OBK / 32; kk++) {
#pragma unroll
        for (int d = D0; d < D1; d++) {
#pragma unroll
            for (int t = (d - S + 1 > 0 ? d - S + 1 : 0); t <= (d < S - 1 ? d : S - 1); t++) {
                const int u = d - t;
                const bool first = kk == 0 && t == (d - S + 1 > 0 ? d - S + 1 : 0);
                mma_i8_any<PAIR>(tmem + (uint32_t)((d - D0) * OBN),
                                 a0 + (uint64_t)(t * (A_TILE >> 4) + kk * 2),
                                 b0 + (uint64_t)(u * (BT >> 4) + kk * 2), (first_kb && first) ? 0u : 1u);
            }
        }
    }
}

// BT: bytes of one digit tile of B in shared memory (128 rows, or the 64 of one CTA of a pair);
// BOFF: offset of the B digit tiles in a stage (after the A digit tiles)
template <int S, bool PAIR = false, int BT = B_TILE, int BOFF = SLOTS * A_TILE>
__device__ __forceinline__ void issue_pass(int p, uint32_t tmem, const uint8_t *st, bool first_kb) {
    const uint64_t a0 = smem_desc_k<64>(st, 0), b0 = smem_desc_k<64>(st + BOFF, 0);
    if (p == 0)
        issue_kblock<S, 0, (S < MAX_DIAG_PER_PASS ? S : MAX_DIAG_PER_PASS), PAIR, BT>(tmem, a0, b0, first_kb);
    else if constexpr (S > MAX_DIAG_PER_PASS)
        issue_kblock<S, MAX_DIAG_PER_PASS, S, PAIR, BT>(tmem, a0, b0, first_kb);
}

template <int S>
__global__ void __launch_bounds__(OTHREADS, 1)
ozaki_gemm_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, OzMap map,
                  int num_tiles) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + OSTAGES * OSTAGE_BYTES);
    uint64_t *empty = full + OSTAGES;
    uint64_t *acc_full = empty + OSTAGES;
    uint64_t *acc_empty = acc_full + 1;
    uint64_t *done = acc_empty + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (threadIdx.x == 0) {
        for (int s = 0; s < OSTAGES; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, OEPI);
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(OTMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            // producer: for every (tile, chunk, pass) unit, the digit tiles of each K block
            int g = 0;
            int issued[OSTAGES] = {};
            for (int t = blockIdx.x; t < num_tiles && !*abort_flag; t += gridDim.x) {
                int m0, n0;
                map.tile(t, m0, n0);
                for (int c = 0; c < map.nchunks && !*abort_flag; c++) {
                    const int kb0 = c * map.kc, kb1 = min(map.nk_all, kb0 + map.kc);
                    for (int p = 0; p < map.npass && !*abort_flag; p++) {
                        int d0, d1, nd;
                        map.pass(p, d0, d1, nd);
                        for (int kb = kb0; kb < kb1; kb++, g++) {
                            const int s = g % OSTAGES;
                            if (!mbar_wait(&empty[s], ((g / OSTAGES) & 1) ^ 1, map.wait_cycles) || *abort_flag) {
                                record_error(map.err, ERR_PRODUCER);
                                *abort_flag = 1;
                                break;
                            }
                            issued[s]++;
                            uint8_t *st = smem + s * OSTAGE_BYTES;
                            mbar_expect_tx(&full[s], (uint32_t)nd * (A_TILE + B_TILE));
                            for (int q = 0; q < nd; q++) {
                                tma_load_3d(&tmA, &full[s], st + q * A_TILE, kb * OBK, m0, q);
                                tma_load_3d(&tmB, &full[s], st + SLOTS * A_TILE + q * B_TILE, kb * OBK, n0, q);
                            }
                        }
                    }
                }
            }
            for (int s = 0; s < OSTAGES; s++)
                if (issued[s] && !mbar_wait(&full[s], (issued[s] - 1) & 1, map.wait_cycles))
                    record_error(map.err, ERR_DRAIN);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer: one unit at a time into the (up to four) diagonal accumulators
            int g = 0, uc = 0;
            for (int t = blockIdx.x; t < num_tiles && !*abort_flag; t += gridDim.x) {
                for (int c = 0; c < map.nchunks && !*abort_flag; c++) {
                    const int kb0 = c * map.kc, kb1 = min(map.nk_all, kb0 + map.kc);
                    for (int p = 0; p < map.npass && !*abort_flag; p++, uc++) {
                        int d0, d1, nd;
                        map.pass(p, d0, d1, nd);
                        if (!mbar_wait(acc_empty, (uc & 1) ^ 1, map.wait_cycles)) {
                            record_error(map.err, ERR_MMA_ACC);
                            *abort_flag = 1;
                            break;
                        }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        for (int kb = kb0; kb < kb1; kb++, g++) {
                            const int s = g % OSTAGES;
                            if (!mbar_wait(&full[s], (g / OSTAGES) & 1, map.wait_cycles) || *abort_flag) {
                                record_error(map.err, ERR_MMA_FULL);
                                *abort_flag = 1;
                                break;
                            }
                            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                            issue_pass<S>(p, tmem, smem + s * OSTAGE_BYTES, kb == kb0);
                            mma_commit(&empty[s]);
                        }
                        mma_commit(acc_full);
                    }
                }
            }
            mma_commit(done);
        }
    } else {
        // epilogue: warp w drains TMEM lanes 32 (w % 4) .. +31, one output row per thread
        const int quarter = warp & 3;
        int uc = 0;
        bool aborted = false;
        for (int t = blockIdx.x; t < num_tiles && !aborted; t += gridDim.x) {
            int m0, n0;
            map.tile(t, m0, n0);
            const int row = m0 + quarter * 32 + lane;
            const double row_scale = row < map.M ? map.alpha * exp2((double)map.ea[row]) : 0.0;
            for (int c = 0; c < map.nchunks && !aborted; c++) {
                for (int p = 0; p < map.npass; p++, uc++) {
                    int d0, d1, nd;
                    map.pass(p, d0, d1, nd);
                    bool ok = !*abort_flag && mbar_wait(acc_full, uc & 1, map.wait_cycles);
                    __syncwarp();
                    if (!ok || *abort_flag) {
                        record_error(map.err, ERR_EPILOGUE);
                        *abort_flag = 1;
                        aborted = true;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const bool first = (c == 0 && p == 0);
                    const uint32_t base = tmem + ((uint32_t)(quarter * 32) << 16);
#pragma unroll 1
                    for (int cc = 0; cc < OBN; cc += 16) {
                        double v[16];
#pragma unroll
                        for (int j = 0; j < 16; j++) v[j] = 0.0;
                        for (int d = d0; d < d1; d++) {
                            uint32_t r[16];
                            tmem_ld16u(base + (uint32_t)((d - d0) * OBN + cc), r);
                            const double w = exp2(-7.0 * (double)(d + 2));
#pragma unroll
                            for (int j = 0; j < 16; j++) v[j] += w * (double)(int)r[j];
                        }
                        if (row < map.M) {
                            double *out = map.C + (long long)(n0 + cc) * map.ldc + row;
                            double old[16];
#pragma unroll
                            for (int j = 0; j < 16; j++) {
                                const bool in = n0 + cc + j < map.N;
                                old[j] = (in && (!first || map.beta != 0.0)) ? __ldcg(out + (long long)j * map.ldc) : 0.0;
                            }
#pragma unroll
                            for (int j = 0; j < 16; j++) {
                                const int col = n0 + cc + j;
                                if (col < map.N) {
                                    const double x = row_scale * exp2((double)map.eb[col]) * v[j];
                                    out[(long long)j * map.ldc] = first ? x + map.beta * old[j] : x + old[j];
                                }
                            }
                        }
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(acc_empty)) : "memory");
                }
            }
        }
    }
    __syncthreads();
    if (!mbar_wait(done, 0, map.wait_cycles)) record_error(map.err, ERR_DONE);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(OTMEM_COLS));
    }
}

// The digit GEMM on a pair of CTAs (a cluster of two): one cta_group::2 MMA of M = 256 (each CTA's
// 128 rows of A) and N = 128 (64 rows of B staged by each CTA).  A 128 x 128 x 32 int8 MMA reads
// 8 KB of operands per 64 tensor cycles, all a single SM's shared memory delivers beside the TMA
// writes; in the pair each SM's shared memory serves its A rows and half of B, 6 KB.  CTA 0 issues
// the MMAs and waits for both CTAs' loads on its own barriers; its commits arrive on both CTAs.
constexpr int BP_TILE = (OBN / 2) * OBK;                         // one CTA's half of a B digit tile

// stages of S-digit operands: S digit tiles of A and S half tiles of B per K block; three stages where
// they fit (up to six digits), which keeps the next two K blocks' loads in flight behind the MMAs
template <int S>
struct PairLayout {
    static constexpr int STAGE = S * (A_TILE + BP_TILE);
    static constexpr int STAGES = 3 * STAGE + 1024 + 256 <= 232448 ? 3 : 2;
    static constexpr int SMEM = STAGES * STAGE + 1024 + 256;
};
static_assert(PairLayout<6>::STAGES == 3 && PairLayout<7>::STAGES == 2, "pair stages");

template <int S>
__global__ void __launch_bounds__(OTHREADS, 1)
ozaki_pair_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, OzMap map,
                  int num_tiles) {
    using PL = PairLayout<S>;
    constexpr int NST = PL::STAGES, STAGE = PL::STAGE, BOFF = S * A_TILE;
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + NST * STAGE);
    uint64_t *empty = full + NST;
    uint64_t *acc_full = empty + NST;
    uint64_t *acc_empty = acc_full + 1;   // used on CTA 0
    uint64_t *done = acc_empty + 1;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = cluster_rank();
    const bool lead = rank == 0;
    const int pair = blockIdx.x >> 1, npairs = gridDim.x >> 1;

    if (threadIdx.x == 0) {
        for (int s = 0; s < NST; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(acc_full, 1);
        mbar_init(acc_empty, 2 * (OEPI / 32));   // one arrival per epilogue warp of each CTA
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(OTMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    cluster_sync();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        if (lane == 0) {
            int g = 0;
            int issued[NST] = {};
            for (int t = pair; t < num_tiles && !*abort_flag; t += npairs) {
                int m0, n0;
                map.tile(t, m0, n0);
                for (int c = 0; c < map.nchunks && !*abort_flag; c++) {
                    const int kb0 = c * map.kc, kb1 = min(map.nk_all, kb0 + map.kc);
                    for (int p = 0; p < map.npass && !*abort_flag; p++) {
                        int d0, d1, nd;
                        map.pass(p, d0, d1, nd);
                        for (int kb = kb0; kb < kb1; kb++, g++) {
                            const int s = g % NST;
                            if (!mbar_wait(&empty[s], ((g / NST) & 1) ^ 1, map.wait_cycles) || *abort_flag) {
                                record_error(map.err, ERR_PRODUCER);
                                *abort_flag = 1;
                                break;
                            }
                            issued[s]++;
                            uint8_t *st = smem + s * STAGE;
                            if (lead) mbar_expect_tx(&full[s], 2u * (uint32_t)nd * (A_TILE + BP_TILE));
                            for (int q = 0; q < nd; q++) {
                                tma_load_3d_pair(&tmA, &full[s], st + q * A_TILE, kb * OBK, m0 + OBM * (int)rank, q);
                                tma_load_3d_pair(&tmB, &full[s], st + BOFF + q * BP_TILE, kb * OBK,
                                                 n0 + (OBN / 2) * (int)rank, q);
                            }
                        }
                    }
                }
            }
            if (lead)
                for (int s = 0; s < NST; s++)
                    if (issued[s] && !mbar_wait(&full[s], (issued[s] - 1) & 1, map.wait_cycles))
                        record_error(map.err, ERR_DRAIN);
        }
    } else if (warp == 1) {
        if (lane == 0 && lead) {
            int g = 0, uc = 0;
            for (int t = pair; t < num_tiles && !*abort_flag; t += npairs) {
                for (int c = 0; c < map.nchunks && !*abort_flag; c++) {
                    const int kb0 = c * map.kc, kb1 = min(map.nk_all, kb0 + map.kc);
                    for (int p = 0; p < map.npass && !*abort_flag; p++, uc++) {
                        if (!mbar_wait(acc_empty, (uc & 1) ^ 1, map.wait_cycles)) {
                            record_error(map.err, ERR_MMA_ACC);
                            *abort_flag = 1;
                            break;
                        }
                        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                        for (int kb = kb0; kb < kb1; kb++, g++) {
                            const int s = g % NST;
                            if (!mbar_wait(&full[s], (g / NST) & 1, map.wait_cycles) || *abort_flag) {
                                record_error(map.err, ERR_MMA_FULL);
                                *abort_flag = 1;
                                break;
                            }
                            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                            issue_pass<S, true, BP_TILE, BOFF>(p, tmem, smem + s * STAGE, kb == kb0);
                            mma_commit_pair(&empty[s]);
                        }
                        mma_commit_pair(acc_full);
                    }
                }
            }
            mma_commit_pair(done);
        }
    } else {
        // epilogue: this CTA's 128 rows; warp w drains TMEM lanes 32 (w % 4) .. +31
        const int quarter = warp & 3;
        int uc = 0;
        bool aborted = false;
        for (int t = pair; t < num_tiles && !aborted; t += npairs) {
            int m0, n0;
            map.tile(t, m0, n0);
            const int row = m0 + OBM * (int)rank + quarter * 32 + lane;
            const double row_scale = row < map.M ? map.alpha * exp2((double)map.ea[row]) : 0.0;
            for (int c = 0; c < map.nchunks && !aborted; c++) {
                for (int p = 0; p < map.npass; p++, uc++) {
                    int d0, d1, nd;
                    map.pass(p, d0, d1, nd);
                    bool ok = !*abort_flag && mbar_wait(acc_full, uc & 1, map.wait_cycles);
                    __syncwarp();
                    if (!ok || *abort_flag) {
                        record_error(map.err, ERR_EPILOGUE);
                        *abort_flag = 1;
                        aborted = true;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const bool first = (c == 0 && p == 0);
                    const uint32_t base = tmem + ((uint32_t)(quarter * 32) << 16);
#pragma unroll 1
                    for (int cc = 0; cc < OBN; cc += 16) {
                        double v[16];
#pragma unroll
                        for (int j = 0; j < 16; j++) v[j] = 0.0;
                        for (int d = d0; d < d1; d++) {
                            uint32_t r[16];
                            tmem_ld16u(base + (uint32_t)((d - d0) * OBN + cc), r);
                            const double w = exp2(-7.0 * (double)(d + 2));
#pragma unroll
                            for (int j = 0; j < 16; j++) v[j] += w * (double)(int)r[j];
                        }
                        if (row < map.M) {
                            double *out = map.C + (long long)(n0 + cc) * map.ldc + row;
                            double old[16];
#pragma unroll
                            for (int j = 0; j < 16; j++) {
                                const bool in = n0 + cc + j < map.N;
                                old[j] = (in && (!first || map.beta != 0.0)) ? __ldcg(out + (long long)j * map.ldc) : 0.0;
                            }
#pragma unroll
                            for (int j = 0; j < 16; j++) {
                                const int col = n0 + cc + j;
                                if (col < map.N) {
                                    const double x = row_scale * exp2((double)map.eb[col]) * v[j];
                                    out[(long long)j * map.ldc] = first ? x + map.beta * old[j] : x + old[j];
                                }
                            }
                        }
                    }
                    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
                    __syncwarp();
                    if (lane == 0) arrive_cta0(acc_empty);
                }
            }
        }
    }
    __syncthreads();
    if (!mbar_wait(done, 0, map.wait_cycles)) record_error(map.err, ERR_DONE);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    cluster_sync();
    if (warp == 1) {
        asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(OTMEM_COLS));
    }
}

// Row exponents of a strided FP64 view (element (r, k) at src[r sr + k sk]): e[r] = the exponent of
// the power of two just above max_k |x_rk| (frexp), by atomicMax over K slices of 32 x 32 tiles
// (e must start below any exponent: all-zero rows keep the start value).
__global__ void oz_rowexp_kernel(const double *__restrict__ src, long long sr, long long sk, int R, int K,
                                 int *__restrict__ e) {
    __shared__ double tile[32][33];
    __shared__ double red[8][33];
    const int r0 = blockIdx.x * 32, tx = threadIdx.x, ty = threadIdx.y;
    const bool k_fast = (sk == 1);
    double m = 0.0;
    for (int k0 = blockIdx.y * 32; k0 < K; k0 += gridDim.y * 32) {
        for (int i = ty; i < 32; i += 8) {
            int r, k;
            if (k_fast) {
                r = r0 + i;
                k = k0 + tx;
            } else {
                r = r0 + tx;
                k = k0 + i;
            }
            const double x = (r < R && k < K) ? src[(long long)r * sr + (long long)k * sk] : 0.0;
            if (k_fast) tile[i][tx] = x;
            else tile[tx][i] = x;
        }
        __syncthreads();
        for (int i = ty; i < 32; i += 8) m = fmax(m, fabs(tile[tx][i]));
        __syncthreads();
    }
    red[ty][tx] = m;
    __syncthreads();
    if (ty == 0 && r0 + tx < R) {
        for (int j = 1; j < 8; j++) m = fmax(m, red[j][tx]);
        if (m > 0.0) {
            int ex;
            frexp(m, &ex);
            atomicMax(&e[r0 + tx], ex);
        }
    }
}

// Digits of the scaled rows: x 2^-e = sum_t d_t 2^(-7(t+1)), d_t = trunc of the remaining fraction
// times 128 (exact in FP64), written as int8 planes [digit][Rp][Kp], K-major, zero padded.
__global__ void oz_digits_kernel(const double *__restrict__ src, long long sr, long long sk, int R, int K, int Rp,
                                 int Kp, int digits, const int *__restrict__ e, int8_t *__restrict__ out) {
    __shared__ double tile[32][33];
    const int r0 = blockIdx.x * 32, tx = threadIdx.x, ty = threadIdx.y;
    const bool k_fast = (sk == 1);
    const size_t plane = (size_t)Rp * Kp;
    for (int k0 = blockIdx.y * 32; k0 < Kp; k0 += gridDim.y * 32) {
        for (int i = ty; i < 32; i += 8) {
            int r, k;
            if (k_fast) {
                r = r0 + i;
                k = k0 + tx;
            } else {
                r = r0 + tx;
                k = k0 + i;
            }
            const double x = (r < R && k < K) ? src[(long long)r * sr + (long long)k * sk] : 0.0;
            if (k_fast) tile[i][tx] = x;
            else tile[tx][i] = x;
        }
        __syncthreads();
        for (int i = ty; i < 32; i += 8) {
            const int r = r0 + i, k = k0 + tx;
            if (r < Rp && k < Kp) {
                const int er = (r < R) ? e[r] : 0;
                double y = (r < R && er > -1100) ? ldexp(tile[i][tx], -er) : 0.0;   // |y| < 1
                const size_t o = (size_t)r * Kp + k;
                for (int t = 0; t < digits; t++) {
                    y *= 128.0;
                    const double d = trunc(y);
                    y -= d;
                    out[t * plane + o] = (int8_t)(int)d;
                }
            }
        }
        __syncthreads();
    }
}

// The same two steps for operands whose K index is contiguous (element (r, k) at src[r sr + k]):
// no transpose is needed, so the rows stream through with 16-byte loads.  One warp per (row, K
// slice) for the exponents; for the digits each thread takes 8 consecutive k of a row and writes one
// 8-byte word per digit plane.
__global__ void oz_rowexp_kfast_kernel(const double *__restrict__ src, long long sr, int R, int K, int kslices,
                                       int *__restrict__ e) {
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    const long long wid = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int per = (K + kslices - 1) / kslices;
    for (long long w = wid; w < (long long)R * kslices; w += nwarps) {
        const int r = (int)(w / kslices), sl = (int)(w - (long long)r * kslices);
        const int k0 = sl * per, k1 = min(K, k0 + per);
        const double *row = src + (long long)r * sr;
        double m = 0.0;
        for (int k = k0 + lane; k < k1; k += 32) m = fmax(m, fabs(__ldg(row + k)));
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (lane == 0 && m > 0.0) {
            int ex;
            frexp(m, &ex);
            atomicMax(&e[r], ex);
        }
    }
}

__global__ void oz_digits_kfast_kernel(const double *__restrict__ src, long long sr, int R, int K, int Rp, int Kp,
                                       int digits, const int *__restrict__ e, int8_t *__restrict__ out) {
    const size_t plane = (size_t)Rp * Kp;
    const int per_row = Kp / 8;
    const long long total = (long long)Rp * per_row;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(idx / per_row), k0 = (int)(idx - (long long)r * per_row) * 8;
        double y[8];
        const int er = r < R ? e[r] : 0;
        const bool live = r < R && er > -1100;
        const double *row = src + (long long)r * sr;
#pragma unroll
        for (int j = 0; j < 8; j++) y[j] = (live && k0 + j < K) ? ldexp(__ldg(row + k0 + j), -er) : 0.0;   // |y| < 1
        int8_t *o = out + (size_t)r * Kp + k0;
        for (int t = 0; t < digits; t++) {
            uint64_t word = 0;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                y[j] *= 128.0;
                const double d = trunc(y[j]);
                y[j] -= d;
                word |= (uint64_t)(uint8_t)(int8_t)(int)d << (8 * j);
            }
            *reinterpret_cast<uint64_t *>(o + t * plane) = word;
        }
    }
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }
inline size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

// digits x rows x Kp tensor of int8, box (64, box_rows, 1), 64-byte swizzle; rows beyond `rows` read
// as zero
CUtensorMap make_i8_map(void *base, int64_t rows, int64_t Kp, int64_t plane_stride, int planes, int box_rows = 128,
                        int64_t row_stride = 0) {
    CUtensorMap m;
    if (row_stride == 0) row_stride = Kp;
    REQUIRE((reinterpret_cast<uintptr_t>(base) & 15) == 0, CCSD_GPU_EINVAL, "tensor map base must be 16-byte aligned");
    REQUIRE(Kp % 64 == 0 && row_stride % 16 == 0 && plane_stride % 16 == 0 && row_stride >= Kp, CCSD_GPU_EINVAL,
            "int8 digit planes: bad padding");
    cuuint64_t dims[3] = {(cuuint64_t)Kp, (cuuint64_t)rows, (cuuint64_t)planes};
    cuuint64_t strides[2] = {(cuuint64_t)row_stride, (cuuint64_t)plane_stride};
    cuuint32_t box[3] = {OBK, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encode_fn()(&m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    REQUIRE(r == CUDA_SUCCESS, CCSD_GPU_ECUDA, "cuTensorMapEncodeTiled (int8) failed: " + std::to_string((int)r));
    return m;
}

int num_sms() {
    int dev = 0, v = 0;
    CU_CHECK(cudaGetDevice(&dev));
    CU_CHECK(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev));
    return v;
}

// exponents e[R] of the rows of a strided view over the whole K
void row_exponents(Exec &ex, const double *src, int64_t sr, int64_t sk, int64_t R, int64_t K, int64_t Rp, int *e) {
    // start every exponent below any frexp exponent: 0x80 bytes = -2139062144
    CU_CHECK(cudaMemsetAsync(e, 0x80, sizeof(int) * (size_t)Rp, ex.stream));
    if (sk == 1) {
        // K slices so that every row has a few warps when rows are few
        const int kslices = (int)std::max<int64_t>(1, std::min<int64_t>((K + 1023) / 1024, (148 * 64 + R - 1) / R));
        const int64_t warps = R * kslices;
        const int blocks = (int)std::min<int64_t>((warps + 7) / 8, 148 * 16);
        oz_rowexp_kfast_kernel<<<blocks, 256, 0, ex.stream>>>(src, sr, (int)R, (int)K, kslices, e);
        ex.launches++;
        CU_CHECK(cudaGetLastError());
        return;
    }
    const int64_t rb = (R + 31) / 32;
    // enough blocks over K to fill the GPU when there are few row blocks
    const int64_t kb = std::max<int64_t>(1, std::min<int64_t>((K + 31) / 32, (4 * 148 + rb - 1) / rb));
    oz_rowexp_kernel<<<dim3((unsigned)rb, (unsigned)std::min<int64_t>(kb, 65535)), dim3(32, 8), 0, ex.stream>>>(
        src, sr, sk, (int)R, (int)K, e);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

// digits [digits][Rp][Kp] of the K slab of a strided view (the exponents are those of whole rows)
void slab_digits(Exec &ex, const double *src, int64_t sr, int64_t sk, int64_t R, int64_t K, int64_t Rp, int64_t Kp,
                 int digits, const int *e, int8_t *out) {
    if (sk == 1) {
        const int64_t total = Rp * (Kp / 8);
        const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 32);
        oz_digits_kfast_kernel<<<blocks, 256, 0, ex.stream>>>(src, sr, (int)R, (int)K, (int)Rp, (int)Kp, digits, e, out);
        ex.launches++;
        CU_CHECK(cudaGetLastError());
        return;
    }
    oz_digits_kernel<<<dim3((unsigned)(Rp / 32), (unsigned)std::min<int64_t>(Kp / 32, 65535)), dim3(32, 8), 0,
                       ex.stream>>>(src, sr, sk, (int)R, (int)K, (int)Rp, (int)Kp, digits, e, out);
    ex.launches++;
    CU_CHECK(cudaGetLastError());
}

}  // namespace

void ozaki_prepare(Exec &ex, bool trans, int64_t rows, int64_t k, const double *X, int64_t ldx, int digits,
                   OzPlanes &out) {
    REQUIRE(rows > 0 && k > 0 && rows < (1ll << 31) && k < (1ll << 31), CCSD_GPU_EINVAL, "ozaki_prepare: bad size");
    REQUIRE(digits >= 2 && digits <= SLOTS, CCSD_GPU_EINVAL, "ozaki_prepare: 2 to 7 digits");
    // rows of op(X): X[r + ldx kk] (N) or X[kk + ldx r] (T), padded to 128 (either operand's tiles)
    const int64_t sr = trans ? ldx : 1, sk = trans ? 1 : ldx;
    const int64_t Rp = round_up(rows, (int64_t)OBM), Kp = round_up(k, (int64_t)OBK);
    const size_t exp_bytes = round_up(sizeof(int) * (size_t)Rp, (size_t)256);
    const size_t need = exp_bytes + (size_t)digits * Rp * Kp;
    if (out.buf.bytes() < need) {
        out.buf.release();
        out.buf.alloc(need, ex.stream);
    }
    out.rows = rows;
    out.k = k;
    out.Rp = Rp;
    out.Kp = Kp;
    out.digits = digits;
    out.exp_bytes = exp_bytes;
    int *e = out.buf.as<int>();
    row_exponents(ex, X, sr, sk, rows, k, Rp, e);
    slab_digits(ex, X, sr, sk, rows, k, Rp, Kp, digits, e, reinterpret_cast<int8_t *>(out.buf.as<uint8_t>() + exp_bytes));
}

void ozaki_gemm(Exec &ex, bool transA, bool transB, int64_t m, int64_t n, int64_t k, double alpha, const double *A,
                int64_t lda, const double *B, int64_t ldb, double beta, double *C, int64_t ldc, int digits,
                const OzPlanes *pa, const OzPlanes *pb) {
    REQUIRE(m > 0 && n > 0 && k > 0, CCSD_GPU_EINVAL, "ozaki_gemm: empty product");
    REQUIRE(!pa || (pa->digits == digits && pa->rows == m && pa->k == k), CCSD_GPU_EINVAL,
            "ozaki_gemm: prepared A does not match");
    REQUIRE(!pb || (pb->digits == digits && pb->rows == n && pb->k == k), CCSD_GPU_EINVAL,
            "ozaki_gemm: prepared B does not match");
    REQUIRE(m < (1ll << 31) && n < (1ll << 31) && k < (1ll << 31), CCSD_GPU_EINVAL, "ozaki_gemm: size too large");
    REQUIRE(digits >= 2 && digits <= SLOTS, CCSD_GPU_EINVAL, "ozaki_gemm: 2 to 7 digits");
    REQUIRE(ex.gemm_err != nullptr, CCSD_GPU_EINVAL, "ozaki_gemm: no error word");
    const int64_t Mp = round_up(m, OBM), Np = round_up(n, OBN);
    // op(A)(r, kk): A[r + lda kk] (N) or A[kk + lda r] (T); op(B)(kk, c) rows c: B[kk + ldb c] (N) or B[c + ldb kk] (T)
    const int64_t a_sr = transA ? lda : 1, a_sk = transA ? 1 : lda;
    const int64_t b_sr = transB ? 1 : ldb, b_sk = transB ? ldb : 1;
    // scratch: exponents of both operands and the digit planes of one K slab
    const size_t exp_bytes = round_up(sizeof(int) * (size_t)(Mp + Np), 256);
    // the digit planes of K slabs of whole 16384-wide chunks, at most ~4 GB of them at a time (a
    // 21 GB operand would otherwise need 18 GB of planes at once); each slab's launch adds its chunks
    // to C in the order one launch over all K would, so the result does not depend on the slabs
    const int64_t per_chunk = (int64_t)digits * std::max<int64_t>(OBM, (pa ? 0 : Mp) + (pb ? 0 : Np)) * OK_CHUNK;
    int64_t budget = 4ll << 30;
    if (const char *mb = std::getenv("CCSD_GPU_DIGIT_SLAB_MB")) budget = std::max<int64_t>(1, std::atoll(mb)) << 20;
    const int64_t chunks_per_slab = std::max<int64_t>(1, budget / per_chunk);
    const int64_t kslab = std::min<int64_t>(round_up(k, OBK), chunks_per_slab * OK_CHUNK);
    const size_t a_bytes = pa ? 0 : round_up((size_t)digits * Mp * kslab, (size_t)1024);
    const size_t b_bytes = pb ? 0 : (size_t)digits * Np * kslab;
    const size_t need = exp_bytes + a_bytes + b_bytes;
    DBuf local;
    DBuf *arena = ex.digit_arena ? ex.digit_arena : &local;
    if (arena->bytes() < need) {
        arena->release();
        arena->alloc(need, ex.stream);
    }
    uint8_t *base = arena->as<uint8_t>();
    int *ea = reinterpret_cast<int *>(base), *eb = ea + Mp;
    int8_t *da = reinterpret_cast<int8_t *>(base + exp_bytes), *db = da + a_bytes;
    // a prepared operand brings its exponents and the digit planes of all of K (no conversion here)
    if (pa) ea = pa->buf.as<int>();
    else row_exponents(ex, A, a_sr, a_sk, m, k, Mp, ea);
    if (pb) eb = pb->buf.as<int>();
    else row_exponents(ex, B, b_sr, b_sk, n, k, Np, eb);
    auto kernel = digits == 7 ? ozaki_gemm_kernel<7> : digits == 6 ? ozaki_gemm_kernel<6>
                : digits == 5 ? ozaki_gemm_kernel<5> : digits == 4 ? ozaki_gemm_kernel<4>
                : digits == 3 ? ozaki_gemm_kernel<3> : ozaki_gemm_kernel<2>;
    auto pkernel = digits == 7 ? ozaki_pair_kernel<7> : digits == 6 ? ozaki_pair_kernel<6>
                 : digits == 5 ? ozaki_pair_kernel<5> : digits == 4 ? ozaki_pair_kernel<4>
                 : digits == 3 ? ozaki_pair_kernel<3> : ozaki_pair_kernel<2>;
    // CTA pairs where 256-row pair tiles pad op(A) no further than 128-row tiles do (10240^3 with 6
    // digits: 18.47 against 18.72 ms; a 528-row operand would run a third of its pair rows empty);
    // CCSD_GPU_PAIR_DIGITS=0 keeps single CTAs
    static const bool pairs_on = [] {
        const char *e = std::getenv("CCSD_GPU_PAIR_DIGITS");
        return !(e && e[0] == '0');
    }();
    const bool pair = pairs_on && m >= 2 * OBM && round_up(m, (int64_t)(2 * OBM)) == Mp;
    CU_CHECK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, OSMEM));
    const int psmem = digits == 7 ? PairLayout<7>::SMEM : digits == 6 ? PairLayout<6>::SMEM
                    : digits == 5 ? PairLayout<5>::SMEM : digits == 4 ? PairLayout<4>::SMEM
                    : digits == 3 ? PairLayout<3>::SMEM : PairLayout<2>::SMEM;
    CU_CHECK(cudaFuncSetAttribute(pkernel, cudaFuncAttributeMaxDynamicSharedMemorySize, psmem));
    const int nsm = num_sms();
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(OTHREADS);
    cfg.dynamicSmemBytes = psmem;
    cfg.stream = ex.stream;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int max_pairs = 1;
    if (pair) {
        static int cached[128] = {};
        int dev = 0;
        CU_CHECK(cudaGetDevice(&dev));
        int &mp = cached[dev & 127];
        if (mp == 0) {
            cfg.gridDim = dim3((unsigned)(2 * (nsm / 2)));
            int n = 0;
            CU_CHECK(cudaOccupancyMaxActiveClusters(&n, pkernel, &cfg));
            mp = std::max(1, n);
        }
        max_pairs = mp;
    }
    for (int64_t k0 = 0; k0 < k; k0 += kslab) {
        const int64_t kk = std::min(kslab, k - k0), Kp = round_up(kk, OBK);
        if (!pa) slab_digits(ex, A + k0 * a_sk, a_sr, a_sk, m, kk, Mp, Kp, digits, ea, da);
        if (!pb) slab_digits(ex, B + k0 * b_sk, b_sr, b_sk, n, kk, Np, Kp, digits, eb, db);
        // prepared planes: the slab starts k0 bytes into each row of the whole-K planes (k0 is a
        // multiple of 16384, so the tensor map base stays 16-byte aligned)
        CUtensorMap ta = pa ? make_i8_map(pa->digits_base() + k0, Mp, Kp, pa->Rp * pa->Kp, digits, OBM, pa->Kp)
                            : make_i8_map(da, Mp, Kp, Mp * Kp, digits);
        CUtensorMap tb = pb ? make_i8_map(pb->digits_base() + k0, Np, Kp, pb->Rp * pb->Kp, digits,
                                          pair ? OBN / 2 : OBN, pb->Kp)
                            : make_i8_map(db, Np, Kp, Np * Kp, digits, pair ? OBN / 2 : OBN);
        OzMap map{};
        map.bm = pair ? 2 * OBM : OBM;
        map.num_mt = (int)(pair ? round_up(Mp, (int64_t)(2 * OBM)) / (2 * OBM) : Mp / OBM);
        map.num_nt = (int)(Np / OBN);
        // raster groups of 2048 rows: their A digit panels (2048 x K x digits bytes) stay in L2 while
        // the group's N tiles stream past
        map.group_m = std::min(map.num_mt, pair ? 8 : 16);
        map.nk_all = (int)(Kp / OBK);
        map.kc = OK_CHUNK / OBK;
        map.nchunks = (map.nk_all + map.kc - 1) / map.kc;
        map.digits = digits;
        map.npass = digits > MAX_DIAG_PER_PASS ? 2 : 1;
        map.M = (int)m;
        map.N = (int)n;
        map.ldc = ldc;
        map.alpha = alpha;
        map.beta = k0 == 0 ? beta : 1.0;
        map.C = C;
        map.ea = ea;
        map.eb = eb;
        map.err = ex.gemm_err;
        map.wait_cycles = ex.wait_cycles > 0 ? ex.wait_cycles : OWAIT_CYCLES;
        const int num_tiles = map.num_mt * map.num_nt;
        const int grid = std::min(num_tiles, pair ? max_pairs : nsm);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (ex.prof && ex.prof->on) {
            CU_CHECK(cudaEventCreate(&e0));
            CU_CHECK(cudaEventCreate(&e1));
            CU_CHECK(cudaEventRecord(e0, ex.stream));
        }
        if (pair) {
            cfg.gridDim = dim3((unsigned)(2 * grid));
            CU_CHECK(cudaLaunchKernelEx(&cfg, pkernel, ta, tb, map, num_tiles));
        } else {
            kernel<<<grid, OTHREADS, OSMEM, ex.stream>>>(ta, tb, map, num_tiles);
            CU_CHECK(cudaGetLastError());
        }
        ex.launches++;
        if (e0) {
            CU_CHECK(cudaEventRecord(e1, ex.stream));
            ex.prof->oz_events.emplace_back(e0, e1);
            ex.prof->oz_ops.push_back(2.0 * (double)digits * (digits + 1) / 2.0 * (double)m * (double)n * (double)kk);
        }
    }
}

int ozaki_products(int digits) { return digits * (digits + 1) / 2; }

}  // namespace ccsd
