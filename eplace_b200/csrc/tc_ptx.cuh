// tc_ptx.cuh -- inline-PTX wrappers of the tcgen05 kernels (tensor-core
// Poisson GEMMs, the network's dense layers): mbarriers, TMA tile loads,
// shared-memory and instruction descriptors of tcgen05.mma (kind::f16, BF16
// operands, FP32 accumulators in tensor memory), tcgen05.ld, and the split of
// an FP32 value into two BF16 planes.  sm_100a only.  No TMA multicast.
#pragma once
#include <cuda.h>

#include <cstdint>

namespace ep {
namespace tc {

constexpr unsigned kWaitLimit = 1u << 22;  // try_wait rounds before giving up

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait of the pipeline (limit: the engine's poll count, kWaitLimit by
// default); returns false (and raises the abort flag) when it gives up or when
// another role already aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort, unsigned limit) {
    for (unsigned it = 0; it < limit; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if (*abort) return false;
    }
    *abort = 1;
    return false;
}

// The wait of the abort path for work this CTA already started (TMA loads
// into its shared memory, MMAs into its TMEM): always kWaitLimit rounds, so
// that a lowered pipeline limit never lets the CTA free TMEM or exit while its
// own copies or MMAs are in flight.
__device__ __forceinline__ void mbar_drain(uint64_t *bar, uint32_t parity) {
    for (unsigned it = 0; it < kWaitLimit && !mbar_try_wait(bar, parity); it++) {
    }
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, uint64_t *bar, int c0,
                                            int c1) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
        : "memory");
}

// UMMA shared-memory descriptor, K-major, 128B swizzle: 8-row x 128 B atoms,
// stride between 8-row groups (SBO) 1024 B, version 1, layout type 2.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)1 << 16;            // LBO (unused for swizzled K-major)
    d |= (uint64_t)(1024 >> 4) << 32;  // SBO
    d |= (uint64_t)1 << 46;            // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;            // SWIZZLE_128B
    return d;
}

// kind::f16 instruction descriptor: D f32, A and B bf16, both K-major.
__host__ __device__ constexpr uint32_t umma_idesc(int m, int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                          uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void bf16_split(float v, uint16_t &hi, uint16_t &lo) {
    uint32_t u = __float_as_uint(v);
    uint32_t r = u + 0x7fffu + ((u >> 16) & 1u);
    hi = (uint16_t)(r >> 16);
    float rem = v - __uint_as_float((uint32_t)hi << 16);
    uint32_t u2 = __float_as_uint(rem);
    lo = (uint16_t)((u2 + 0x7fffu + ((u2 >> 16) & 1u)) >> 16);
}

}  // namespace tc
}  // namespace ep
