// cs_ptx.cuh — inline-PTX building blocks for the sm_100a compaction kernels:
// mbarrier phase tracking, 1-D TMA bulk copies (cp.async.bulk, no multicast),
// relaxed GPU-scope accesses for the look-back status words, and a bounded wait
// helper built on %globaltimer.
#pragma once
#include <cstdint>

namespace cs {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Programmatic dependent launch: block until the grids this one depends on (the previous
// kernels on the stream) have completed and their memory is visible. A no-op when the
// kernel was launched without programmatic stream serialization.
__device__ __forceinline__ void grid_dependency_wait()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// ---------------------------------------------------------------------------------
// mbarrier (CTA scope)
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t tx_bytes)
{
    asm volatile(
        "{\n\t.reg .b64 st;\n\t"
        "mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(smem_u32(bar)),
        "r"(tx_bytes)
        : "memory");
}

// One probe of the phase with the given parity. True once that phase has completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
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

// Bounded wait: returns false if the phase did not complete within timeout_ns.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint64_t timeout_ns)
{
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > timeout_ns) return false;
    }
}

#ifndef CS_SUSPEND_NS
#define CS_SUSPEND_NS 250000u
#endif
// One probe that may suspend the thread in hardware (up to CS_SUSPEND_NS) until the phase
// completes, so waiting warps do not spin on the issue slots.
__device__ __forceinline__ bool mbar_try_wait_suspend(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(CS_SUSPEND_NS)
        : "memory");
    return ok != 0;
}

// Warp-uniform bounded wait (call with all 32 lanes). Every lane probes (each performs its
// own acquire); the warp leaves together once all lanes saw the phase complete, or together
// with `false` once the time bound ran out. A lane that already saw completion keeps
// seeing it: the phase cannot advance again before this warp has done its part of the
// next one.
__device__ __forceinline__ bool mbar_wait_warp(uint64_t* bar, uint32_t parity, uint64_t timeout_ns, uint32_t lane)
{
    (void)lane;
    if (__all_sync(0xffffffffu, mbar_try_wait_suspend(bar, parity))) return true;
    const uint64_t t0 = globaltimer_ns();
    while (true) {
        if (__all_sync(0xffffffffu, mbar_try_wait_suspend(bar, parity))) return true;
        if (__any_sync(0xffffffffu, globaltimer_ns() - t0 > timeout_ns)) return false;
    }
}

// ---------------------------------------------------------------------------------
// TMA bulk copy global -> shared (1-D, non-tensor, no multicast). Both addresses
// 16-byte aligned, size a multiple of 16. Completion is signalled as transaction bytes
// on the mbarrier.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void bulk_g2s(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Same, with an L2 eviction-priority hint (streaming payload: evict-first).
__device__ __forceinline__ uint64_t l2_policy_evict_first()
{
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ void bulk_g2s_hint(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar,
                                              uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::"r"(
            smem_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// ---------------------------------------------------------------------------------
// GPU-scope relaxed accesses for the look-back status words (flag and value share one
// 64-bit word, so no further ordering is needed for the protocol itself).
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t ld_relaxed_gpu(const uint64_t* p)
{
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_relaxed_gpu(uint64_t* p, uint64_t v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t ld_relaxed_gpu_u32(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Read-only streaming loads (never written by the same kernel).
__device__ __forceinline__ uint32_t ldg_u32(const uint32_t* p)
{
    return __ldg(p);
}

// ---------------------------------------------------------------------------------
// Shared-memory vector access
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint4 lds128(const void* p)
{
    return *reinterpret_cast<const uint4*>(p);
}

__device__ __forceinline__ void sts128(void* p, uint4 v)
{
    *reinterpret_cast<uint4*>(p) = v;
}

// Streaming 128-bit global store (evict-first: the output is not re-read).
__device__ __forceinline__ void stg128_cs(void* p, uint4 v)
{
    __stcs(reinterpret_cast<uint4*>(p), v);
}

// ---------------------------------------------------------------------------------
// Warp scans
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, uint32_t lane)
{
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint32_t t = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= (uint32_t)d) v += t;
    }
    return v;
}

__device__ __forceinline__ uint64_t warp_incl_scan64(uint64_t v, uint32_t lane)
{
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint64_t t = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= (uint32_t)d) v += t;
    }
    return v;
}

__device__ __forceinline__ uint64_t warp_sum64(uint64_t v)
{
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}

__device__ __forceinline__ uint32_t warp_sum32(uint32_t v)
{
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}

} // namespace cs
