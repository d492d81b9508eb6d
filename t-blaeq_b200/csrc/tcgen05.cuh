// Thin inline-PTX wrappers for the sm_100a tensor-core path shared by the k-means assignment and
// the frontier scorer: shared-memory matrix and instruction descriptors, mbarriers with bounded
// waits, bulk copies, tensor-memory allocation and loads, and single-CTA tcgen05.mma.
#pragma once

#include <cstdint>

namespace tblaeq {
namespace tc {

__device__ __forceinline__ uint32_t smemAddr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (sm100 version 1) of a K-major, non-swizzled operand image of
// 8-row x 16-byte core matrices: `lbo` = bytes between core matrices adjacent in K, `sbo` = bytes
// between 8-row groups.
__device__ __forceinline__ uint64_t smemDesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((saddr & 0x3FFFFu) >> 4) | (static_cast<uint64_t>(lbo >> 4) << 16) |
           (static_cast<uint64_t>(sbo >> 4) << 32) | (1ull << 46);
}

// Operand formats of the instruction descriptor: BF16 under kind::f16, TF32 under kind::tf32.
constexpr uint32_t kFmtBf16 = 1;
constexpr uint32_t kFmtTf32 = 2;

// Instruction descriptor: D = F32 (bits 4-5 = 1), A and B of format `fmt` (bits 7-9, 10-12), both
// K-major, N / 8 at bits 17-22, M / 16 at bits 24-28.
constexpr uint32_t instrDesc(uint32_t fmt, uint32_t M, uint32_t N) {
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

// ---- mbarriers ----------------------------------------------------------------------------------
__device__ __forceinline__ void mbarInit(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}
// Makes mbarrier initialisations visible to the async proxy (bulk copies, tcgen05.commit).
__device__ __forceinline__ void mbarInitFence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbarExpectTx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbarArrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}
__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smemAddr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// Waits for the phase with parity `phase` to complete, at most `limit` polls; false when it gave up.
__device__ __forceinline__ bool mbarWait(uint64_t* bar, uint32_t phase, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbarTryWait(bar, phase)) return true;
    return false;
}

// ---- copies and fences --------------------------------------------------------------------------
// Bulk copy global -> shared (16-byte aligned addresses, size a multiple of 16), completing on `bar`.
__device__ __forceinline__ void bulkLoad(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smemAddr(dst)),
                 "l"(src), "r"(bytes), "r"(smemAddr(bar))
                 : "memory");
}
// Orders this thread's ordinary shared-memory writes before later tensor-core reads of them.
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tcFenceBefore() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tcFenceAfter() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// ---- tensor memory ------------------------------------------------------------------------------
// One warp allocates `cols` columns (a power of two >= 32) and writes their address to `slot`; the
// CTA gives up its right to allocate again, so other CTAs on the SM are never kept waiting.
__device__ __forceinline__ void tmemAlloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smemAddr(slot)), "r"(cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmemDealloc(uint32_t taddr, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(cols) : "memory");
}
// 32 consecutive 32-bit columns of the calling thread's lane (warp w reads lanes 32(w%4)..+31).
__device__ __forceinline__ void tmemLoad32(uint32_t taddr, uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmemWaitLoad() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---- MMA ----------------------------------------------------------------------------------------
enum Kind { kKindF16, kKindTf32 };

// D[tmem] (+)= A[smem] x B[smem]^T, issued by one thread; `accumulate` = 0 overwrites D.
template <Kind K>
__device__ __forceinline__ void mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                    uint32_t accumulate) {
    if constexpr (K == kKindTf32) {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
    } else {
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
            "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
            : "memory");
    }
}
// Arrives once on `bar` when every MMA this thread issued so far has completed.
__device__ __forceinline__ void mmaCommit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smemAddr(bar))
                 : "memory");
}

}  // namespace tc
}  // namespace tblaeq
