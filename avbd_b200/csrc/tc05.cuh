// tc05.cuh -- the pieces of the sm_100a tensor-core path used by the MLP
// kernels, as inline PTX: tcgen05.mma (kind::f16, BF16 operands from shared
// memory, FP32 accumulator in tensor memory), tcgen05.commit to an mbarrier,
// bounded mbarrier waits, TMEM allocation and tcgen05.ld.
//
// Operand layout: K-major, no swizzle.  A matrix of R rows (M or N) by K BF16
// elements is stored as "core matrices" of 8 rows x 8 elements (16 bytes per
// row, 128 contiguous bytes); with K chunks of 8 elements outermost,
//     byte(r, k) = (k / 8) * (R * 16) + r * 16 + (k % 8) * 2,
// the descriptor's stride byte offset (between 8-row groups) is 128 and its
// leading byte offset (between K chunks) is R * 16.  One MMA consumes K = 16
// (two chunks); the next K step starts 2 * R * 16 bytes further.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace avbd {
namespace tc {

AVBD_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) of an R-row K-major operand
AVBD_HD constexpr uint32_t kmaj_off(uint32_t r, uint32_t k, uint32_t R) {
    return (k >> 3) * (R * 16u) + r * 16u + (k & 7u) * 2u;
}

// shared-memory matrix descriptor (sm_100 format: version 1, no swizzle)
AVBD_D uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor, kind::f16: D F32, A and B BF16, both K-major, dense
AVBD_HD constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one K = 16 step; issued by a single thread
AVBD_D void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

// the mbarrier receives one arrival when all earlier MMAs of this thread are done
AVBD_D void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

AVBD_D void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

AVBD_D bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete; gives up after
// `limit` polls (each poll may suspend the thread for a while) and returns
// false, so a kernel can record an error instead of hanging.
AVBD_D bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = 1u << 22) {
    for (uint32_t i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// TMEM allocation: executed by all 32 threads of one warp
AVBD_D void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols)
                 : "memory");
}
AVBD_D void tmem_relinquish() { asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory"); }
AVBD_D void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

AVBD_D void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
AVBD_D void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core
AVBD_D void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes
// 32 (w % 4) .. +31); the wait is in the same statement so no use of the
// registers can be scheduled before the data has arrived.
AVBD_D void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace avbd
