// cs_pattern.cu — compaction by a periodic pattern instead of a mask in memory.
//
// Element i is selected when bit (i % L) of `pattern` is set (LSB-first, 1 <= L <= 32). With
// P = popcount of the pattern's L bits, output j is input (j / P) * L + pos[j % P], pos[r]
// being the r-th set bit: every output has a closed-form source, so there is no popcount
// pass, no scan and no mask read. Each thread produces 16-byte output vectors (16 / w
// consecutive outputs, streaming stores) and gathers their sources with read-only loads;
// neighbouring lanes read neighbouring periods, so the loads of a warp fall on few lines
// and DRAM reads each touched sector once. A thread keeps the loads of 16 outputs in flight
// before it stores, and the (quotient, remainder) of the output index advances
// incrementally, so a thread divides once.
// Reference: bench9_pattern (src/benchmarks.cuh:397-416) over launch_pattern_proc /
// kernel_pattern_proc (src/kernels/kernel_pattern.cuh:13-131), whose pattern is read from
// the most significant bit (element i <-> bit 31 - i % L); pass __brev of such a pattern.
#include <cstdint>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"

namespace cs {

namespace {

template <typename T, bool VEC_OUT>
__global__ void __launch_bounds__(256) k_pattern(const T* __restrict__ in, T* __restrict__ out, uint32_t pattern,
                                                 uint32_t L, uint32_t P, uint64_t count, uint64_t* d_count)
{
    constexpr uint32_t VEC = 16 / sizeof(T);
    __shared__ uint32_t s_pos[32];
    if (threadIdx.x < 32) {
        const uint32_t b = threadIdx.x;
        if (b < L && ((pattern >> b) & 1u)) s_pos[__popc(pattern & ((1u << b) - 1u))] = b;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_count = count;
    __syncthreads();
    const uint64_t nvec = (count + VEC - 1) / VEC;
    const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    // a thread takes UNR vectors stride apart per iteration, all their loads before any store;
    constexpr uint32_t UNR = sizeof(T); // 16 elements per iteration at every width
    const uint64_t dq1 = (stride * VEC) / P; // output-index step between a thread's vectors
    const uint32_t dr1 = static_cast<uint32_t>((stride * VEC) % P);
    uint64_t q = (tid * VEC) / P;
    uint32_t r = static_cast<uint32_t>((tid * VEC) % P);
    for (uint64_t v0 = tid; v0 < nvec; v0 += UNR * stride) {
        union {
            uint4 u;
            T e[VEC];
        } x[UNR];
        uint64_t qk = q;
        uint32_t rk = r;
#pragma unroll
        for (uint32_t k = 0; k < UNR; ++k) {
            const uint64_t j0 = (v0 + k * stride) * VEC;
            uint64_t qq = qk;
            uint32_t rr = rk;
#pragma unroll
            for (uint32_t e = 0; e < VEC; ++e) {
                x[k].e[e] = j0 + e < count ? __ldg(in + qq * L + s_pos[rr]) : T(0);
                if (++rr == P) {
                    rr = 0;
                    ++qq;
                }
            }
            qk += dq1;
            rk += dr1;
            if (rk >= P) {
                rk -= P;
                ++qk;
            }
        }
#pragma unroll
        for (uint32_t k = 0; k < UNR; ++k) {
            const uint64_t j0 = (v0 + k * stride) * VEC;
            if (j0 >= count) break;
            if (VEC_OUT && j0 + VEC <= count) {
                stg128_cs(out + j0, x[k].u);
            } else {
#pragma unroll
                for (uint32_t e = 0; e < VEC; ++e)
                    if (j0 + e < count) out[j0 + e] = x[k].e[e];
            }
        }
        q = qk; // the next iteration's first vector is UNR strides on
        r = rk;
    }
}

template <typename T>
cudaError_t launch_t(const void* in, void* out, uint32_t pattern, uint32_t L, uint32_t P, uint64_t count,
                     uint64_t* d_count, int sms, cudaStream_t s)
{
    constexpr uint64_t VEC = 16 / sizeof(T);
    const uint64_t nvec = (count + VEC - 1) / VEC;
    uint64_t blocks = (nvec + 255) / 256;
    const uint64_t cap = static_cast<uint64_t>(sms) * 8;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    const bool vec = (reinterpret_cast<uintptr_t>(out) & 15u) == 0;
    const T* ti = static_cast<const T*>(in);
    T* to = static_cast<T*>(out);
    if (vec)
        k_pattern<T, true><<<static_cast<unsigned>(blocks), 256, 0, s>>>(ti, to, pattern, L, P, count, d_count);
    else
        k_pattern<T, false><<<static_cast<unsigned>(blocks), 256, 0, s>>>(ti, to, pattern, L, P, count, d_count);
    note_launch();
    return cudaGetLastError();
}

} // namespace

uint64_t pattern_count(uint64_t n, uint32_t pattern, uint32_t L)
{
    const uint32_t pm = L >= 32 ? pattern : (pattern & ((1u << L) - 1u));
    const uint32_t rem = static_cast<uint32_t>(n % L);
    const uint32_t partial = rem ? (pm & ((1u << rem) - 1u)) : 0u;
    return (n / L) * static_cast<uint64_t>(__builtin_popcount(pm)) + static_cast<uint64_t>(__builtin_popcount(partial));
}

} // namespace cs

using namespace cs;

extern "C" {

int compressstore_pattern(const void* d_in, void* d_out, uint64_t n, uint32_t elem_bytes, uint32_t pattern,
                          uint32_t pattern_length, uint64_t* d_count, cs_stream_t stream)
{
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8) return CS_ERR_INVALID_VALUE;
    if (pattern_length < 1 || pattern_length > 32 || !d_count) return CS_ERR_INVALID_VALUE;
    if (n > (1ull << 40) - 1) return CS_ERR_NOT_SUPPORTED;
    if (reinterpret_cast<uintptr_t>(d_count) & 7u) return CS_ERR_MISALIGNED;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint32_t pm = pattern_length >= 32 ? pattern : (pattern & ((1u << pattern_length) - 1u));
    const uint64_t count = pattern_count(n, pm, pattern_length);
    if (count == 0) {
        const cudaError_t e = cudaMemsetAsync(d_count, 0, sizeof(uint64_t), s);
        return e == cudaSuccess ? CS_SUCCESS : CS_ERR_CUDA;
    }
    if (!d_in || !d_out) return CS_ERR_INVALID_VALUE;
    if ((reinterpret_cast<uintptr_t>(d_in) | reinterpret_cast<uintptr_t>(d_out)) & (elem_bytes - 1u))
        return CS_ERR_MISALIGNED;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return CS_ERR_NO_DEVICE;
    const uint32_t P = static_cast<uint32_t>(__builtin_popcount(pm));
    cudaError_t e;
    switch (elem_bytes) {
        case 1: e = launch_t<uint8_t>(d_in, d_out, pm, pattern_length, P, count, d_count, sms, s); break;
        case 2: e = launch_t<uint16_t>(d_in, d_out, pm, pattern_length, P, count, d_count, sms, s); break;
        case 4: e = launch_t<uint32_t>(d_in, d_out, pm, pattern_length, P, count, d_count, sms, s); break;
        default: e = launch_t<uint64_t>(d_in, d_out, pm, pattern_length, P, count, d_count, sms, s); break;
    }
    return e == cudaSuccess ? CS_SUCCESS : (e == cudaErrorMemoryAllocation ? CS_ERR_OUT_OF_MEMORY : CS_ERR_CUDA);
}

} // extern "C"
