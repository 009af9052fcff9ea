// Bulk asynchronous copies (TMA, cp.async.bulk) between global and shared
// memory, completed on an mbarrier, for sm_100a.  Every wait is bounded: a
// wait that runs out of iterations records an error code in the plan's
// status word (mapped host memory, read through sfl_plan_status and checked
// by the next call on the plan) and gives up instead of spinning forever.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace sfl {

// Status codes written to a plan's device status word (0 = fine).
constexpr int kStatusMbarTimeout = 1;
constexpr long long kMbarSpinLimit = 1LL << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("{ .reg .b64 st; mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1; }" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Raises the barrier's expected transaction bytes without arriving: a thread
// that issues a copy announces its bytes first, so the count cannot reach
// zero before the copy completes.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("{ .reg .b64 st; mbarrier.arrive.shared::cta.b64 st, [%0]; }" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Waits for `phase` of the barrier with an iteration limit; false on timeout
// (*status then holds kStatusMbarTimeout).  The status word is mapped host
// memory: a plain store, made visible to the host by a system-scope fence.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, int* status,
                                                  long long limit = kMbarSpinLimit) {
    for (long long it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    *reinterpret_cast<volatile int*>(status) = kStatusMbarTimeout;
    __threadfence_system();
    return false;
}

// global -> shared, `bytes` a multiple of 16, both addresses 16-byte aligned.
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// shared -> global, bulk-group completion.
__device__ __forceinline__ void bulk_store(void* gmem_dst, const void* smem_src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gmem_dst), "r"(smem_u32(smem_src)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }



// Waits until this thread's committed bulk stores have read shared memory.
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// Makes this thread's generic-proxy shared-memory writes visible to later
// bulk copies (async proxy).
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace sfl
