// Device-side helpers: shared-memory addressing, mbarriers, 1-D bulk copies
// (cp.async.bulk, the TMA engine's untiled mode), the per-device status word
// and small launch utilities.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "mv_internal.h"

namespace mv {

// Iteration bound for every spin on an mbarrier.  A healthy bulk copy lands in
// microseconds; this bound is seconds, and exceeding it raises
// MV_DEV_WAIT_TIMEOUT instead of hanging the GPU.
constexpr uint32_t kWaitSpinLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// 1-D bulk copy global -> shared (no multicast).  dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// The waits take the barrier as a shared-memory address (32-bit) or as a pointer into shared memory.
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    return mbar_try_wait(smem_u32(bar), parity);
}

// Bounded wait; returns false (and raises MV_DEV_WAIT_TIMEOUT) on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, uint32_t *status, uint32_t limit) {
    for (uint32_t it = 0; it < limit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    if (status) atomicOr(status, MV_DEV_WAIT_TIMEOUT);
    return false;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t *status,
                                                  uint32_t limit) {
    return mbar_wait_bounded(smem_u32(bar), parity, status, limit);
}

// 4-byte asynchronous copy global -> shared (cp.async, no registers): src_bytes (0, 2 or 4) are read, the
// rest of the 4 bytes is zero-filled.  dst and src 4-byte aligned.  Completion: cp_async_commit, then
// cp_async_wait_all in the issuing thread (and a barrier for other threads).
__device__ __forceinline__ void cp_async_4(void *dst, const void *src, uint32_t src_bytes) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// 16-byte asynchronous copy global -> shared (dst a shared-memory address), cached in L2 only; dst and src
// 16-byte aligned.
__device__ __forceinline__ void cp_async_16(uint32_t dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
// Arrive on an mbarrier (shared-memory address) once every cp.async this thread issued so far has landed,
// without raising the barrier's expected count: the barrier's arrival count must include one arrival per
// thread that calls this.
__device__ __forceinline__ void cp_async_mbar_arrive_noinc(uint32_t bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ uint4 ldg_nc_u4(const uint4 *p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

// Host side: per-device status word, lazily allocated once per device.
uint32_t *device_status_word(mv_status *st);
uint32_t wait_spin_limit();   // kWaitSpinLimit unless MV_INJECT_WAIT_LIMIT set another bound
int inject_drop_copy();
int sm_count();
int max_smem_optin();
int max_smem_per_sm();
// Raise the kernel's dynamic shared-memory limit to `smem` (once per kernel
// and device) and, if blocks_per_sm is non-NULL, return its occupancy for
// `threads` threads (cached).  Safe to call while a stream is being captured.
mv_status prepare_kernel(const void *kern, size_t smem, int threads, int *blocks_per_sm);

inline mv_status cuda_fail(cudaError_t e, const char *what) {
    return fail(MV_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define MV_CUDA_TRY(expr, what)                              \
    do {                                                     \
        cudaError_t _e = (expr);                             \
        if (_e != cudaSuccess) return mv::cuda_fail(_e, what); \
    } while (0)

}  // namespace mv
