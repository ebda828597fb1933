// TMA bulk copies (cp.async.bulk, global -> shared) completed on a shared-memory mbarrier, with
// bounded waits. Used to stage the basis/quadrature tables of a kernel in shared memory once per
// CTA. The source is always this GPU's own memory (tables uploaded at context creation); no
// cluster multicast is used.
//
// Rules the callers keep: both addresses 16-byte aligned, sizes multiples of 16 bytes, the
// transaction count of one phase below 2^20 bytes.
#pragma once
#include <cstdint>

namespace fvedg {

// Polls of a bulk-copy wait before it gives up (each try_wait may suspend the thread briefly).
constexpr long long kBulkSpinLimit = 1ll << 20;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the async (TMA) proxy before any copy names it
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also announces `bytes` of transactions for the current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}

// Waits for phase `parity` of the barrier at most `limit` polls; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, long long limit) {
    for (long long i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Thread 0 of the CTA: copies `bytes` from src to dst in chunks of at most 16 KB, all on one phase
// of `bar` (announced beforehand by mbar_arrive_expect_tx with the total).
__device__ __forceinline__ void bulk_copy_chunks(void* dst, const void* src, size_t bytes, uint64_t* bar) {
    constexpr size_t kChunk = 16384;
    for (size_t o = 0; o < bytes; o += kChunk) {
        const size_t n = bytes - o < kChunk ? bytes - o : kChunk;
        bulk_copy_g2s(static_cast<char*>(dst) + o, static_cast<const char*>(src) + o, (unsigned)n, bar);
    }
}

}  // namespace fvedg
