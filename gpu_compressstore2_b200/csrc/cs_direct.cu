// cs_direct.cu — the 1-pass form for short columns: one CTA per 4096-element tile, no
// warp specialisation, no TMA pipeline.
//
// For a short column the persistent TMA kernel is latency-bound: its chain per unit (ticket,
// mask copy, popcount, look-back, payload copy, placement, store) runs once or twice per CTA
// and the pipeline set-up is not amortised (2^20 uint32: 13.8 us per launch in ncu, 44% of
// SM cycles active). Here every thread loads its 16 elements and their 16 mask bits straight
// into registers, the CTA scans the counts, takes its output offset by a CTA-wide decoupled
// look-back over the tile statuses (256 predecessors per round, lookback_cta), places the
// selected elements in a shared-memory stage at their output alignment and writes the tile's
// run with 16-byte stores. Tiles are taken in order from an atomic ticket, so a tile only
// waits on tiles already held by running CTAs; every wait is bounded.
//
// Reference: the same operation as kernel_3pass_proc_true_striding_optimized_writeout
// (src/kernels/kernel_3pass.cuh:329-467) with its popcount and prefix passes
// (kernel_3pass.cuh:12-214) folded into one launch.
#include <cstdint>
#include <cuda_runtime.h>

#include "cs_internal.cuh"

namespace cs {

namespace {

constexpr uint32_t DT_THREADS = 256;
constexpr uint32_t DT_EPT = 16;                          // elements per thread
constexpr uint32_t DT_TILE = DT_THREADS * DT_EPT;        // 4096 elements per tile
static_assert(DT_TILE == DIRECT_TILE_ELEMS, "tile size shared with the host");

template <typename T>
__global__ void __launch_bounds__(DT_THREADS) k_compact_direct(const CompactParams p)
{
    constexpr uint32_t VEC = 16 / sizeof(T); // elements per 16-byte vector
    constexpr uint32_t NV = DT_EPT / VEC;    // vectors per thread
    __shared__ __align__(16) T stage[DT_TILE + VEC];
    __shared__ LookbackSmem<DT_THREADS / 32> s_lb;
    __shared__ uint32_t s_warp[DT_THREADS / 32];
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_flag;
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5;
    grid_dependency_wait(); // an earlier call may still use this workspace
    const ColumnDesc& C = p.col0;
    const uint64_t n = C.n;
    const uint32_t epoch = p.hdr->epoch;
    const T* __restrict__ in = reinterpret_cast<const T*>(C.in);
    T* __restrict__ out = reinterpret_cast<T*>(C.out);

    while (true) {
        if (tid == 0) s_tile = atomicAdd(&p.hdr->tile_counter, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= p.num_tiles) break;
        // this thread's 16 elements and their mask bits (bits at positions >= n are dropped)
        const uint64_t e0 = tile * DT_TILE + static_cast<uint64_t>(tid) * DT_EPT;
        uint32_t bits = 0;
        union {
            uint4 v[NV];
            T e[DT_EPT];
        } x;
        if (e0 < n) {
            bits = (__ldg(C.mask + e0 / 32) >> (e0 & 31u)) & 0xffffu;
            if (e0 + DT_EPT > n) bits &= (1u << (n - e0)) - 1u;
            if (e0 + DT_EPT <= n) {
                const uint4* src = reinterpret_cast<const uint4*>(in + e0);
#pragma unroll
                for (uint32_t v = 0; v < NV; ++v) x.v[v] = __ldg(src + v);
            } else {
#pragma unroll
                for (uint32_t k = 0; k < DT_EPT; ++k) x.e[k] = e0 + k < n ? in[e0 + k] : T(0);
            }
        }
        // exclusive scan of the counts over the CTA
        const uint32_t c = __popc(bits);
        const uint32_t incl = warp_incl_scan(c, lane);
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        uint32_t wbase = 0, total = 0;
#pragma unroll
        for (uint32_t w = 0; w < DT_THREADS / 32; ++w) {
            const uint32_t v = s_warp[w];
            wbase += w < warp ? v : 0u;
            total += v;
        }
        const uint32_t excl = wbase + incl - c;
        uint64_t prefix = lookback_cta<DT_THREADS>(p.status, tile, total, epoch, p.timeout_ns, p.hdr, s_lb);
        if (prefix != POISON && prefix + total > n) {
            if (tid == 0) record_error(p.hdr, DEVERR_RANGE);
            prefix = POISON;
        }
        if (tile == p.num_tiles - 1 && tid == 0) *C.d_count = prefix == POISON ? POISON : prefix + total;
        if (prefix != POISON) {
            // stage index a + i holds output element prefix + i, a = prefix % VEC, so the
            // stage's 16-byte vectors map to aligned 16-byte runs of the output
            const uint32_t a = static_cast<uint32_t>(prefix % VEC);
            uint32_t pos = a + excl;
#pragma unroll
            for (uint32_t k = 0; k < DT_EPT; ++k) {
                if ((bits >> k) & 1u) stage[pos] = x.e[k];
                pos += (bits >> k) & 1u;
            }
            __syncthreads();
            T* gdst = out + (prefix - a);
            const uint32_t end = a + total;
            const uint32_t nvec = (end + VEC - 1) / VEC;
            for (uint32_t v = tid; v < nvec; v += DT_THREADS) {
                const uint32_t s0 = v * VEC, s1 = s0 + VEC;
                if (s0 >= a && s1 <= end) {
                    stg128_cs(gdst + s0, lds128(stage + s0));
                } else {
                    const uint32_t lo = s0 > a ? s0 : a, hi = s1 < end ? s1 : end;
                    for (uint32_t e = lo; e < hi; ++e) gdst[e] = stage[e];
                }
            }
        }
        __syncthreads(); // the stage and s_warp are rewritten by the next tile
    }
    lookback_kernel_epilogue(p.hdr, &p.hdr->tile_counter, &p.hdr->done_counter, &s_flag, false, p.keep_begin,
                             p.keep_end);
}

template <typename T>
cudaError_t launch_t(const CompactParams& p, int num_sms, cudaStream_t stream)
{
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_compact_direct<T>, DT_THREADS, 0);
    if (e != cudaSuccess) return e;
    uint64_t grid = static_cast<uint64_t>(per_sm < 1 ? 1 : per_sm) * static_cast<uint64_t>(num_sms);
    if (grid > p.num_tiles) grid = p.num_tiles;
    if (grid == 0) grid = 1;
    e = launch_pdl(k_compact_direct<T>, dim3(static_cast<unsigned>(grid)), dim3(DT_THREADS), 0, stream, p);
    note_launch();
    return e;
}

} // namespace

cudaError_t launch_compact_direct(const CompactParams& p, uint32_t elem_bytes, int num_sms, cudaStream_t stream)
{
    switch (elem_bytes) {
        case 1: return launch_t<uint8_t>(p, num_sms, stream);
        case 2: return launch_t<uint16_t>(p, num_sms, stream);
        case 4: return launch_t<uint32_t>(p, num_sms, stream);
        case 8: return launch_t<uint64_t>(p, num_sms, stream);
        default: return cudaErrorInvalidValue;
    }
}

} // namespace cs
