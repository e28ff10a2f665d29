// Bulk asynchronous copies (the TMA engine's 1-D form, cp.async.bulk) from
// global into shared memory, completed on an mbarrier, for sm_100a. Used to
// stage the next work item's contiguous particle ranges and terrain rows
// while the current one is computed. Only this GPU's own memory is ever a
// source, and no copy is multicast.
//
// Rules of the instruction that the callers keep: source and destination
// 16-byte aligned, size a positive multiple of 16; a thread that issues copies
// into a buffer first orders the CTA's earlier ordinary accesses of it with
// fence_proxy_async(); every wait is bounded.
#pragma once

#include <cuda.h>  // CUtensorMap

#include <cstdint>

namespace slab {
namespace tma {

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// before the barrier's shared memory is used for anything else (all waits done)
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// make the initialised barriers visible to the async proxy
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// order the CTA's earlier ordinary shared-memory accesses (after a barrier)
// before later bulk copies into the same bytes
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// one arrival that also announces `bytes` of copies to come
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_addr(bar)),
        "r"(bytes)
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of the barrier, at most `limit` polls (each poll
// itself suspends for a while in hardware). Returns false if it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit = 1 << 22) {
    for (int k = 0; k < limit; ++k)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// bytes (a multiple of 16) from global src to shared dst (both 16-byte
// aligned), completing on bar
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// A box of a 2-D tensor (map built on the host by cuTensorMapEncodeTiled)
// into shared memory (128-byte aligned), completing on bar. x is the inner
// coordinate in elements; x times the element size must be a multiple of 16.
// The map is a __grid_constant__ kernel parameter; no multicast.
__device__ __forceinline__ void tensor_g2s_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

}  // namespace tma

// Per-thread asynchronous copies global -> shared (cp.async): a thread
// requests many small copies without holding the values in registers, so a
// whole work item's gather goes out in one round. Each copy is 4, 8 or 16
// bytes with both addresses aligned to its size; wait_all() completes the
// thread's own copies, and a CTA barrier after it shows them to the others.
namespace cpa {

__device__ __forceinline__ void copy4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(tma::smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void copy8(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(tma::smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void copy16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(tma::smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

}  // namespace cpa
}  // namespace slab
