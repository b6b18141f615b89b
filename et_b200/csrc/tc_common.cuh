// Device helpers shared by the tcgen05 GEMM kernels of libccsd_gpu (sm_100a): shared-memory
// addresses, mbarriers with bounded waits, TMA tile loads, UMMA shared-memory descriptors,
// tcgen05 commit and TMEM loads, the CTA-pair (cta_group::2) forms of loads, commits and arrivals,
// and the driver entry point that encodes TMA tensor maps.
#pragma once

#include <cuda.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "common.cuh"

namespace ccsd {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// the first bounded wait that runs out names the error; later ones keep it
__device__ __forceinline__ void record_error(int *err, int code) { atomicCAS(err, 0, code); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// bounded wait for the completion of the phase with the given parity; false after `limit` cycles
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit) {
    uint32_t addr = smem_u32(bar);
    const long long t0 = clock64();
    while (true) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > limit) return false;
    }
}

__device__ __forceinline__ void tma_load_3d(const CUtensorMap *map, uint64_t *bar, void *dst, int c0, int c1,
                                            int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// K-major operand tile of rows of `row_bytes` bytes (128 or 64) stored contiguously by TMA with the
// matching swizzle: 8-row atoms stacked along M/N, so the stride byte offset is 8 rows; the leading
// byte offset is unused for swizzled K-major layouts.  Layout types: SWIZZLE_128B = 2,
// SWIZZLE_64B = 4 (bits 61-63 of the sm_100 descriptor, version 1 in bits 46-47).
template <int ROW_BYTES>
__device__ __forceinline__ uint64_t smem_desc_k(const void *tile, uint32_t k_byte_offset) {
    static_assert(ROW_BYTES == 128 || ROW_BYTES == 64, "row bytes");
    const uint64_t addr = smem_u32(tile) + k_byte_offset;
    uint64_t d = 0;
    d |= (addr >> 4) & 0x3FFFull;                          // start address
    d |= (uint64_t)(16 >> 4) << 16;                        // leading byte offset
    d |= (uint64_t)((8 * ROW_BYTES) >> 4) << 32;           // stride byte offset
    d |= 1ull << 46;                                       // descriptor version (sm_100)
    d |= (uint64_t)(ROW_BYTES == 128 ? 2 : 4) << 61;       // SWIZZLE_128B / SWIZZLE_64B
    return d;
}

// 128-byte swizzle (the bf16 kernel's 64-element K rows)
__device__ __forceinline__ uint64_t smem_desc(const void *tile, uint32_t k_byte_offset) {
    return smem_desc_k<128>(tile, k_byte_offset);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16u(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// ---- CTA pairs (a cluster of two CTAs sharing cta_group::2 MMAs) ----
constexpr uint32_t PEER_BIT_CLEAR = 0xFEFFFFFFu;   // shared::cluster address of the same offset in CTA 0

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// tile load into this CTA's shared memory whose bytes complete on CTA 0's barrier
__device__ __forceinline__ void tma_load_3d_pair(const CUtensorMap *map, uint64_t *bar, void *dst, int c0, int c1,
                                                 int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, "
        "%5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar) & PEER_BIT_CLEAR), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// arrives on the barrier at this offset in both CTAs once the pair's MMAs issued so far complete
__device__ __forceinline__ void mma_commit_pair(uint64_t *bar) {
    asm volatile(
        "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 [%0], %1;" ::"r"(
            smem_u32(bar)),
        "h"((uint16_t)3)
        : "memory");
}

__device__ __forceinline__ void arrive_cta0(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cluster.b64 _, [%0];" ::"r"(smem_u32(bar) & PEER_BIT_CLEAR) : "memory");
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda)
inline EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    REQUIRE(fn != nullptr, CCSD_GPU_ECUDA, "cuTensorMapEncodeTiled unavailable");
    return fn;
}

}  // namespace tc
}  // namespace ccsd
