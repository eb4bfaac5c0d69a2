// Thin inline-PTX wrappers for the sm_90+/sm_100a asynchronous data movement used by the
// kernels: mbarrier phases, the bulk (TMA engine) global->shared copy, and 4-byte cp.async.
// Every copy has exactly one destination CTA: this one.
#pragma once

#include <cstdint>

namespace tsk {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

// Makes the initialised barriers visible to the async proxy (bulk copies complete on them).
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("{\n\t.reg .b64 st;\n\t"
                 "mbarrier.arrive.release.cta.shared::cta.b64 st, [%0];\n\t}" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

// One bounded probe of the phase with the given parity; true once it has completed. The
// thread may be suspended until the phase completes, for at most about kSuspendNs, so a waiting
// warp issues few instructions.
constexpr uint32_t kSuspendNs = 2000;
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2, %3;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(smem_addr(bar)), "r"(parity), "n"(kSuspendNs)
                 : "memory");
    return done != 0;
}

// Waits with an iteration limit (at most about 2^21 x 2 us); false when the limit was reached
// (the caller reports it).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    constexpr uint32_t kLimit = 1u << 21;
    for (uint32_t i = 0; i < kLimit; ++i) {
        if (mbar_try_wait(bar, parity)) {
            return true;
        }
    }
    return false;
}

// For a waiter with slack (the producer, stages ahead of its consumers): probes without a
// suspend hint and sleeps between probes, so that a long wait costs few issue slots. Bounded
// like mbar_wait (at most about 2^20 probes of at most ~1 us each).
__device__ __forceinline__ bool mbar_wait_backoff(uint64_t *bar, uint32_t parity) {
    constexpr uint32_t kLimit = 1u << 20;
    for (uint32_t i = 0; i < kLimit; ++i) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(smem_addr(bar)), "r"(parity)
                     : "memory");
        if (done != 0) {
            return true;
        }
        __nanosleep(256);
    }
    return false;
}

// Bulk copy of bytes (multiple of 16, both addresses 16-byte aligned) from global memory into
// this CTA's shared memory; completion is signalled as transaction bytes on bar.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1], %2, [%3];" ::"r"(smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// 4-byte asynchronous copy global -> shared (both 4-byte aligned).
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src)
                 : "memory");
}

// 16-byte asynchronous copy global -> shared (both 16-byte aligned), in this thread's current
// cp.async group; commit closes the group, wait<N> waits until at most N groups are pending.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The barrier receives one more arrival once all of this thread's earlier cp.async copies have
// landed (the pending count is raised first, so the phase cannot complete before them).
__device__ __forceinline__ void cp_async_arrive(uint64_t *bar) {
    asm volatile("cp.async.mbarrier.arrive.shared::cta.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// Programmatic dependent launch. wait: blocks until the grids this one depends on in its
// stream have completed and their memory is visible (immediately when the launch had no
// programmatic dependency). launch_dependents: lets the next grid of the stream start its
// prologue once every CTA of this grid has issued it or exited.
__device__ __forceinline__ void griddep_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void griddep_launch_dependents() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Named barrier over a subset of the CTA's warps. The id is an immediate: a barrier id known
// only at run time makes the compiler reserve all sixteen barriers for the kernel, and the
// barriers a CTA reserves bound how many CTAs an SM holds.
template <uint32_t Id> __device__ __forceinline__ void named_sync(uint32_t threads) {
    static_assert(Id < 16, "sixteen hardware barriers");
    asm volatile("bar.sync %0, %1;" ::"n"(Id), "r"(threads) : "memory");
}

// The same with the id in a register: the kernel then reserves all sixteen barriers, which
// limits an SM to four CTAs (64 barriers per SM). Used where that limit is the intent.
__device__ __forceinline__ void named_sync_any(uint32_t id, uint32_t threads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

// Barrier 1 + group for one of Groups groups of warps (barriers 1 .. Groups). Groups = 0: the
// id in a register (named_sync_any).
template <uint32_t Groups>
__device__ __forceinline__ void group_sync(uint32_t group, uint32_t threads) {
    static_assert(Groups <= 8, "at most eight groups");
    if constexpr (Groups == 0) {
        named_sync_any(1 + group, threads);
        return;
    }
    switch (group) {
    case 0: named_sync<1>(threads); break;
    case 1: if constexpr (Groups > 1) named_sync<2>(threads); break;
    case 2: if constexpr (Groups > 2) named_sync<3>(threads); break;
    case 3: if constexpr (Groups > 3) named_sync<4>(threads); break;
    case 4: if constexpr (Groups > 4) named_sync<5>(threads); break;
    case 5: if constexpr (Groups > 5) named_sync<6>(threads); break;
    case 6: if constexpr (Groups > 6) named_sync<7>(threads); break;
    default: if constexpr (Groups > 7) named_sync<8>(threads); break;
    }
}

// 16-byte store to global memory (an evict-first hint measured slower). No memory clobber: the
// kernel never reads what it stores.
__device__ __forceinline__ void st_global_v4(void *p, uint32_t a, uint32_t b, uint32_t c,
                                             uint32_t d) {
    asm volatile("st.global.v4.b32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(a), "r"(b), "r"(c),
                 "r"(d));
}

__device__ __forceinline__ uint4 ld_nc_v4(const void *p) {
    uint4 v;
    asm volatile("ld.global.nc.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

} // namespace tsk
