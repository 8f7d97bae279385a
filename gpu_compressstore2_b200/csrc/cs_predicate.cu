// cs_predicate.cu — pass 0 of predicate compaction: the selection mask is computed from
// the payload on the device instead of being read (k_pred_mask). The 3-pass form then runs
// on that mask: k_popc_blocks (chunk counts and prefixes), the sparse gather and the
// TMA-staged writeout.
// Reference: the reference evaluates the predicate on the host while packing the mask
// (gen_predicate, src/utils.cuh:102-122, with predicate_function x > threshold,
// src/main.cu:24-28,92) and copies mask and payload to the device before compacting.
#include <cstdint>
#include <cstring>

#include <atomic>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"

namespace cs {

namespace {

template <typename T>
__device__ __forceinline__ T from_bits(uint64_t b)
{
    T v;
    memcpy(&v, &b, sizeof(T)); // little-endian: the low bytes hold the value
    return v;
}

// The comparison of each cs_pred_op as one instruction where it can be; lo/hi are the
// host-prepared bounds (LT/LE: hi = a; GT/GE/EQ/NE: lo = a; BETWEEN: lo = a, hi = b). Every
// ordered comparison with a NaN is false, != is true (C++ semantics).
template <int OP, typename T>
__device__ __forceinline__ bool pred_eval(T x, T lo, T hi)
{
    if constexpr (OP == CS_PRED_LT) return x < hi;
    else if constexpr (OP == CS_PRED_LE) return x <= hi;
    else if constexpr (OP == CS_PRED_GT) return x > lo;
    else if constexpr (OP == CS_PRED_GE) return x >= lo;
    else if constexpr (OP == CS_PRED_EQ) return x == lo;
    else if constexpr (OP == CS_PRED_NE) return x != lo;
    else return lo <= x && x <= hi;
}

// Mask words from the payload: a grid-stride pass in which every thread takes UNR 16-byte
// vectors (16 / w elements each) per iteration, all loads before the evaluation; the
// G = 32 / (16 / w) lanes that share a mask word OR their shifted bits with xor shuffles and
// one of them stores the word. Bits at positions >= n are zero.
// 16-byte vectors per thread per iteration, and whether the grid is one resident wave.
// Measured on B200 (us per compressstore_if call, one wave vs a grid of 8 CTAs per SM, of
// which only the resident ones run at first): 2^28 f32 497 -> 468 (UNR 4; 8: 467), 2^28 u64
// 1170 -> 938 (UNR 8; 4: 1073), but 2^29 u8 463 -> 467 and u16 585 -> 594, whose per-element
// evaluation keeps the old grid busy. With the bounds-free path, UNR 8 on the old grid:
// u8 428.5 -> 425.7, u16 579.0 -> 553.9 (one wave with UNR 8: 431.0 / 560.8).
template <typename T>
struct PredShape {
    static constexpr uint32_t UNR = sizeof(T) == 4 ? 4u : 8u;
    static constexpr bool ONE_WAVE = sizeof(T) >= 4;
};

template <typename T, int OP>
__global__ void __launch_bounds__(256) k_pred_mask(const PredParams pp)
{
    constexpr uint32_t VEC = 16 / sizeof(T); // elements per lane load
    constexpr uint32_t G = 32 / VEC;         // lanes per mask word
    constexpr uint32_t UNR = PredShape<T>::UNR;
    const uint32_t lane = threadIdx.x & 31u;
    const T lo = from_bits<T>(pp.lo), hi = from_bits<T>(pp.hi);
    grid_dependency_wait(); // an earlier call may still read this mask buffer
    const uint64_t n = pp.bs.col0.n;
    const uint64_t nw = (n + 31) / 32;
    const uint64_t nvec = (n + VEC - 1) / VEC;
    const T* __restrict__ in = reinterpret_cast<const T*>(pp.in);
    uint32_t* __restrict__ mask = pp.mask;
    // warps stride over groups of 32 vectors; a thread's vector is (group * 32 + lane)
    const uint64_t warp_global = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t total_warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const uint64_t ngroups = (nvec + 31) / 32;
    const uint4* __restrict__ in4 = reinterpret_cast<const uint4*>(pp.in);
    const uint64_t vstride = total_warps * 32;  // vectors between a thread's consecutive groups
    const uint64_t wstride = total_warps * VEC; // mask words between them
    const uint32_t sh = (lane * VEC) & 31u;
    for (uint64_t g0 = warp_global; g0 < ngroups; g0 += UNR * total_warps) {
        union {
            uint4 u;
            T e[VEC];
        } x[UNR];
        if ((g0 + (UNR - 1) * total_warps + 1) * 32 * VEC <= n) {
            // every group of this iteration is complete: no per-element bounds or tail bits
            const uint4* src = in4 + g0 * 32 + lane;
#pragma unroll
            for (uint32_t k = 0; k < UNR; ++k) x[k].u = __ldg(src + k * vstride);
            uint32_t* dst = mask + g0 * VEC + lane / G;
#pragma unroll
            for (uint32_t k = 0; k < UNR; ++k) {
                uint32_t bits = 0;
#pragma unroll
                for (uint32_t i = 0; i < VEC; ++i) bits |= static_cast<uint32_t>(pred_eval<OP>(x[k].e[i], lo, hi)) << i;
                uint32_t m = bits << sh;
#pragma unroll
                for (uint32_t d = 1; d < G; d <<= 1) m |= __shfl_xor_sync(0xffffffffu, m, d);
                if ((lane % G) == 0u) dst[k * wstride] = m;
            }
            continue;
        }
#pragma unroll
        for (uint32_t k = 0; k < UNR; ++k) {
            const uint64_t v = (g0 + k * total_warps) * 32 + lane;
            const uint64_t e0 = v * VEC;
            if (e0 + VEC <= n) {
                x[k].u = __ldg(reinterpret_cast<const uint4*>(in) + v);
            } else {
#pragma unroll
                for (uint32_t i = 0; i < VEC; ++i) x[k].e[i] = e0 + i < n ? in[e0 + i] : T(0);
            }
        }
#pragma unroll
        for (uint32_t k = 0; k < UNR; ++k) {
            const uint64_t g = g0 + k * total_warps;
            if (g >= ngroups) break; // warp-uniform
            uint32_t bits = 0;
#pragma unroll
            for (uint32_t i = 0; i < VEC; ++i) bits |= static_cast<uint32_t>(pred_eval<OP>(x[k].e[i], lo, hi)) << i;
            if ((g + 1) * 32 * VEC > n) { // the last group: clear bits at positions >= n
                const uint64_t e0 = (g * 32 + lane) * VEC;
                bits &= e0 >= n ? 0u : (e0 + VEC <= n ? 0xffffffffu : ((1u << (n - e0)) - 1u));
            }
            uint32_t m = bits << ((lane * VEC) & 31u);
#pragma unroll
            for (uint32_t d = 1; d < G; d <<= 1) m |= __shfl_xor_sync(0xffffffffu, m, d);
            const uint64_t word = g * VEC + lane / G; // a group of 32 vectors covers VEC words
            if ((lane % G) == 0u && word < nw) mask[word] = m;
        }
    }
}

// CTAs of k_pred_mask<T, OP> resident on one SM at once (taken once). For 4- and 8-byte
// elements the grid-stride pass is launched as one wave of them: CTAs beyond it would run
// their whole share after the first wave finished, with a fraction of the bytes in flight.
template <typename T, int OP>
int pred_resident_per_sm()
{
    static std::atomic<int> cached{0};
    int v = cached.load(std::memory_order_relaxed);
    if (v > 0) return v;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_pred_mask<T, OP>, 256, 0) != cudaSuccess || v < 1) {
        cudaGetLastError();
        v = 4;
    }
    cached.store(v, std::memory_order_relaxed);
    return v;
}

template <typename T, int OP>
cudaError_t launch_op(const PredParams& pp, int num_sms, cudaStream_t stream)
{
    constexpr uint64_t VEC = 16 / sizeof(T);
    const uint64_t nvec = (pp.bs.col0.n + VEC - 1) / VEC;
    constexpr uint64_t UNR = PredShape<T>::UNR;
    uint64_t blocks = (nvec + 256 * UNR - 1) / (256 * UNR); // one iteration per thread
    const uint64_t per_sm = PredShape<T>::ONE_WAVE ? static_cast<uint64_t>(pred_resident_per_sm<T, OP>()) : 8u;
    const uint64_t cap = static_cast<uint64_t>(num_sms) * per_sm;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    return launch_pdl(k_pred_mask<T, OP>, dim3(static_cast<unsigned>(blocks)), dim3(256), 0, stream, pp);
}

template <typename T>
cudaError_t launch_t(const PredParams& pp, int op, int num_sms, cudaStream_t stream)
{
    switch (op) {
        case CS_PRED_LT: return launch_op<T, CS_PRED_LT>(pp, num_sms, stream);
        case CS_PRED_LE: return launch_op<T, CS_PRED_LE>(pp, num_sms, stream);
        case CS_PRED_GT: return launch_op<T, CS_PRED_GT>(pp, num_sms, stream);
        case CS_PRED_GE: return launch_op<T, CS_PRED_GE>(pp, num_sms, stream);
        case CS_PRED_EQ: return launch_op<T, CS_PRED_EQ>(pp, num_sms, stream);
        case CS_PRED_NE: return launch_op<T, CS_PRED_NE>(pp, num_sms, stream);
        default: return launch_op<T, CS_PRED_BETWEEN>(pp, num_sms, stream);
    }
}

} // namespace

cudaError_t launch_pred_mask(const PredParams& pp, int type, int op, int num_sms, cudaStream_t stream)
{
    cudaError_t e;
    switch (type) {
        case CS_U8: e = launch_t<uint8_t>(pp, op, num_sms, stream); break;
        case CS_U16: e = launch_t<uint16_t>(pp, op, num_sms, stream); break;
        case CS_U32: e = launch_t<uint32_t>(pp, op, num_sms, stream); break;
        case CS_U64: e = launch_t<uint64_t>(pp, op, num_sms, stream); break;
        case CS_I8: e = launch_t<int8_t>(pp, op, num_sms, stream); break;
        case CS_I16: e = launch_t<int16_t>(pp, op, num_sms, stream); break;
        case CS_I32: e = launch_t<int32_t>(pp, op, num_sms, stream); break;
        case CS_I64: e = launch_t<int64_t>(pp, op, num_sms, stream); break;
        case CS_F32: e = launch_t<float>(pp, op, num_sms, stream); break;
        case CS_F64: e = launch_t<double>(pp, op, num_sms, stream); break;
        default: return cudaErrorInvalidValue;
    }
    note_launch();
    return e;
}

} // namespace cs
