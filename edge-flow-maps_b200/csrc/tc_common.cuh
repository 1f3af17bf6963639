// Blackwell (sm_100a) tensor-core primitives in inline PTX: UMMA shared-memory
// and instruction descriptors, tcgen05.mma (BF16 x BF16 -> FP32, one CTA),
// TMEM allocation and loads, and mbarrier waits that give up after a bounded
// number of polls.
//
// Operands use the canonical "interleaved" (SWIZZLE_NONE) shared-memory
// layouts of the UMMA descriptors:
//   K-major : core matrix = 8 rows (M or N) x 8 K-elements, 128 contiguous
//             bytes (row r at +16 r); row groups SBO bytes apart, the two
//             8-element K halves of one K=16 instruction LBO bytes apart;
//   MN-major: core matrix = 8 K-rows x 8 M/N-elements (16 bytes along M/N,
//             K-row j at +16 j); M/N groups SBO bytes apart, K groups LBO
//             bytes apart.
#pragma once
#include <cstdint>

#include "edge_common.cuh"

namespace tc {

EDGE_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start address, leading / stride byte
// offsets (all >> 4, 14 bits), version 1, base offset 0, SWIZZLE_NONE
EDGE_HD uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor of kind::f16 with BF16 A and B, FP32 accumulator;
// a_mn / b_mn select MN-major operands
EDGE_HD uint32_t idesc_bf16(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
EDGE_D void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t accumulate) {
    uint32_t z = 0;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t"
        "}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(z), "r"(z), "r"(z), "r"(z));
}

// arrive on the mbarrier once all previously issued MMAs of this thread complete
EDGE_D void commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}

EDGE_D void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// wait for the phase with the given parity; false if it did not complete
// within max_polls polls (each poll suspends for a bounded time)
EDGE_D bool mbar_wait(uint32_t mbar, uint32_t parity, int max_polls) {
    for (int i = 0; i < max_polls; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t"
            ".reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t"
            "}\n"
            : "=r"(ok)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// expect `bytes` of asynchronous copies on mbar (one arrival)
EDGE_D void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// bulk copy (TMA, no tensor map, no multicast) of `bytes` (a multiple of 16,
// both addresses 16-byte aligned) from global memory into this CTA's shared
// memory, completion counted on mbar
EDGE_D void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"((unsigned long long)__cvta_generic_to_global(src)), "r"(bytes), "r"(mbar)
        : "memory");
}

// generic-proxy shared-memory writes -> visible to the tensor cores
EDGE_D void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
EDGE_D void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
EDGE_D void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TMEM columns (power of two >= 32), allocated and freed by one whole warp
EDGE_D void tmem_alloc(uint32_t slot_saddr, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot_saddr), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
EDGE_D void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes
// 32w..32w+31; taddr carries the lane in bits 16+)
EDGE_D void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; q++) v[q] = __uint_as_float(r[q]);
}

}  // namespace tc
