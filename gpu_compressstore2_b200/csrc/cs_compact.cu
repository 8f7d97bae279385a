// cs_compact.cu — the TMA-staged, warp-specialised persistent compaction kernel.
//
// One CTA per SM walks tiles of TILE_BYTES payload (TILE_BYTES/w elements) through an
// S-stage shared-memory ring:
//   warp 0  producer : takes the next tile id (device counter for the 1-pass form, static
//                      round robin for the 3-pass form) and issues 1-D TMA bulk copies
//                      (cp.async.bulk, no multicast) of the tile's mask words and payload
//                      into stage s; the ragged last tile is topped up with plain loads.
//   warp 1  scanner  : popcounts the tile's mask words, scans them into per-compute-warp
//                      bases, obtains the tile's output offset (decoupled look-back in the
//                      1-pass form, the pass-2 chunk offset in the 3-pass form) and
//                      publishes it to the compute warps.
//   warps 2.. compute: each owns TILE_BYTES/NCW contiguous bytes of the tile. Lanes read
//                      16-byte payload vectors from shared memory, place the selected
//                      elements in a per-warp staging buffer at their output positions
//                      (popc of the mask bits below them, shuffled per word), release the
//                      stage, then emit the staged run with 16-byte streaming stores;
//                      only the ragged head/tail vectors are written element by element.
//
// Reference: kernel_3pass_proc_true_striding_optimized_writeout
// (src/kernels/kernel_3pass.cuh:329-467) stages 32 source indices per warp and gathers
// from global memory; the popcount and prefix passes it depends on are
// src/kernels/kernel_3pass.cuh:12-214. Every wait is bounded (timeout_ns) and leaves the
// kernel through the normal exit path with an error recorded in the workspace header.
#include <cstdint>
#include <cuda_runtime.h>

#include "cs_internal.cuh"

namespace cs {

constexpr int NCW = 8;                  // compute warps
constexpr int NWARPS = NCW + 2;         // + producer + scanner
constexpr int NTHREADS = NWARPS * 32;
constexpr int STAGES = 4;

template <int NC>
struct TileMeta {
    int64_t tile;          // -1: end of work
    uint64_t prefix;       // output offset of the tile (POISON: do not write)
    uint32_t warp_base[NC];
    uint32_t total;
    uint32_t pad;
};

template <typename T, int S, int NC>
struct Layout {
    static constexpr uint32_t TE = TILE_BYTES / sizeof(T); // tile elements
    static constexpr uint32_t W = TE / 32;                  // mask words per tile
    static constexpr uint32_t MASK_BYTES = W * 4;
    static constexpr uint32_t SEG_BYTES = TILE_BYTES / NC;  // bytes per compute warp
    static constexpr uint32_t STAGE_OUT_BYTES = SEG_BYTES + 16;
    static constexpr uint32_t PAY = 0;
    static constexpr uint32_t MASK = PAY + S * TILE_BYTES;
    static constexpr uint32_t OUTB = MASK + S * MASK_BYTES;
    static constexpr uint32_t META = OUTB + NC * STAGE_OUT_BYTES;
    static constexpr uint32_t BARS = (META + S * sizeof(TileMeta<NC>) + 15u) & ~15u;
    static constexpr uint32_t TOTAL = BARS + 4 * S * 8;
    static_assert(MASK_BYTES % 16 == 0, "mask stage must keep 16-byte alignment");
    static_assert(SEG_BYTES % 16 == 0 && (TE / NC) % 32 == 0, "segments must be whole words and vectors");
    static_assert(W % 128 == 0, "scanner reads 4 words per lane step");
};

template <typename T, int MODE, int S, int NC>
__global__ void __launch_bounds__(NTHREADS, 1) k_compact_tma(const CompactParams p)
{
    using L = Layout<T, S, NC>;
    constexpr uint32_t TE = L::TE;
    constexpr uint32_t W = L::W;
    constexpr uint32_t VEC = 16 / sizeof(T);         // elements per 16-byte vector
    constexpr uint32_t E = TE / NC;                  // elements per compute warp
    constexpr uint32_t SW = E / 32;                  // mask words per compute warp
    constexpr uint32_t WPP = SW < 32 ? SW : 32;      // words per pass
    constexpr uint32_t PASSES = SW / WPP;
    constexpr uint32_t GROUPS = WPP / VEC;           // 32*VEC-element groups per pass
    constexpr uint32_t LPW_SCAN = 32 / NC;           // scanner lanes per compute warp
    constexpr uint32_t KWORDS = W / 32;              // mask words per scanner lane
    static_assert(SW % WPP == 0 && WPP % VEC == 0, "pass/group shape");

    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint32_t s_flag;
    uint8_t* pay = smem + L::PAY;
    uint32_t* msk = reinterpret_cast<uint32_t*>(smem + L::MASK);
    uint8_t* outb = smem + L::OUTB;
    TileMeta<NC>* meta = reinterpret_cast<TileMeta<NC>*>(smem + L::META);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::BARS);
    uint64_t* full_mask = bars;
    uint64_t* full_pay = bars + S;
    uint64_t* ready = bars + 2 * S;
    uint64_t* empty = bars + 3 * S;

    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31u;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full_mask[s], 1);
            mbar_init(&full_pay[s], 1);
            mbar_init(&ready[s], 32);
            mbar_init(&empty[s], NC * 32);
        }
        fence_mbar_init();
    }
    __syncthreads();
    const uint32_t epoch = (MODE == 0) ? p.hdr->epoch : 0u;
    const bool scan_ok = (MODE == 1) ? last_scan_ok(p.hdr) : true; // 3-pass: pass 2 completed cleanly

    if (warp == 0) {
        // ------------------------------------------------------------- producer
        const uint64_t policy = l2_policy_evict_first();
        uint32_t j = 0;
        for (;; ++j) {
            const uint32_t s = j % S;
            const uint32_t u = j / S;
            if (u > 0 && !mbar_wait_warp(&empty[s], (u - 1) & 1u, p.timeout_ns, lane)) {
                if (lane == 0) record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                break;
            }
            uint64_t tile;
            if (MODE == 0) {
                uint32_t t = 0;
                if (lane == 0) t = atomicAdd(&p.hdr->tile_counter, 1u);
                tile = __shfl_sync(0xffffffffu, t, 0);
            } else {
                tile = static_cast<uint64_t>(blockIdx.x) + static_cast<uint64_t>(j) * gridDim.x;
            }
            if (tile >= p.num_tiles) {
                if (lane == 0) {
                    meta[s].tile = -1;
                    mbar_arrive(&full_mask[s]);
                    mbar_arrive(&full_pay[s]);
                }
                ++j;
                break;
            }
            const uint64_t e0 = tile * TE;
            const uint64_t rem = p.n - e0;
            if (lane == 0) meta[s].tile = static_cast<int64_t>(tile);
            if (rem >= TE) {
                if (lane == 0) {
                    mbar_arrive_expect_tx(&full_mask[s], L::MASK_BYTES);
                    bulk_g2s(msk + s * W, p.mask + tile * W, L::MASK_BYTES, &full_mask[s]);
                    mbar_arrive_expect_tx(&full_pay[s], TILE_BYTES);
                    bulk_g2s_hint(pay + s * TILE_BYTES, p.in + tile * TILE_BYTES, TILE_BYTES, &full_pay[s], policy);
                }
            } else {
                // ragged last tile: mask words by plain loads (zero past n), payload bulk
                // copy of the 16-byte-multiple part plus byte loads of the remainder
                const uint64_t nw = (p.n + 31) / 32;
                const uint64_t w0 = tile * W;
                for (uint32_t i = lane; i < W; i += 32) {
                    const uint64_t wi = w0 + i;
                    uint32_t m = 0;
                    if (wi < nw) {
                        m = __ldg(p.mask + wi);
                        if (wi == nw - 1 && (p.n & 31u)) m &= (1u << (p.n & 31u)) - 1u;
                    }
                    msk[s * W + i] = m;
                }
                const uint32_t bytes = static_cast<uint32_t>(rem) * static_cast<uint32_t>(sizeof(T));
                const uint32_t aligned = bytes & ~15u;
                for (uint32_t b = aligned + lane; b < bytes; b += 32)
                    pay[s * TILE_BYTES + b] = __ldg(p.in + tile * TILE_BYTES + b);
                __syncwarp();
                if (lane == 0) {
                    __threadfence_block();
                    mbar_arrive(&full_mask[s]);
                    if (aligned) {
                        mbar_arrive_expect_tx(&full_pay[s], aligned);
                        bulk_g2s_hint(pay + s * TILE_BYTES, p.in + tile * TILE_BYTES, aligned, &full_pay[s], policy);
                    } else {
                        mbar_arrive(&full_pay[s]);
                    }
                }
            }
        }
        // Drain: the most recent arming of each stage must have landed before the CTA may
        // exit (normally already true; matters only after a timeout).
        for (uint32_t k = 0; k < (uint32_t)S && k < j; ++k) {
            const uint32_t jj = j - 1 - k;
            mbar_wait_warp(&full_mask[jj % S], (jj / S) & 1u, p.timeout_ns, lane);
            mbar_wait_warp(&full_pay[jj % S], (jj / S) & 1u, p.timeout_ns, lane);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------- scanner
        for (uint32_t j = 0;; ++j) {
            const uint32_t s = j % S;
            const uint32_t u = j / S;
            if (!mbar_wait_warp(&full_mask[s], u & 1u, p.timeout_ns, lane)) {
                if (lane == 0) record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                break;
            }
            const int64_t tile = meta[s].tile;
            if (tile < 0) {
                mbar_arrive(&ready[s]);
                break;
            }
            const uint32_t* mw = msk + s * W + lane * KWORDS;
            uint32_t c = 0;
#pragma unroll
            for (uint32_t i = 0; i < KWORDS; i += 4) {
                const uint4 q = lds128(mw + i);
                c += __popc(q.x) + __popc(q.y) + __popc(q.z) + __popc(q.w);
            }
            const uint32_t incl = warp_incl_scan(c, lane);
            const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
            if ((lane % LPW_SCAN) == 0) meta[s].warp_base[lane / LPW_SCAN] = incl - c;
            uint64_t prefix;
            if (MODE == 0) {
                prefix = lookback_warp(p.status, static_cast<uint64_t>(tile), total, epoch, p.timeout_ns, p.hdr, lane);
            } else {
                prefix = scan_ok ? p.chunk_offsets[(static_cast<uint64_t>(tile) * TE) >> p.chunk_log2] : POISON;
            }
            if (prefix != POISON && prefix + total > p.n) {
                if (lane == 0) record_error(p.hdr, DEVERR_RANGE);
                prefix = POISON;
            }
            if (lane == 0) {
                meta[s].prefix = prefix;
                meta[s].total = total;
                if (MODE == 0 && static_cast<uint64_t>(tile) == p.num_tiles - 1)
                    *p.d_count = (prefix == POISON) ? POISON : prefix + total;
            }
            __syncwarp();
            mbar_arrive(&ready[s]);
        }
    } else {
        // ------------------------------------------------------------- compute
        const uint32_t cw = warp - 2;
        T* stage = reinterpret_cast<T*>(outb + cw * L::STAGE_OUT_BYTES);
        for (uint32_t j = 0;; ++j) {
            const uint32_t s = j % S;
            const uint32_t u = j / S;
            if (!mbar_wait_warp(&ready[s], u & 1u, p.timeout_ns, lane)) {
                if (lane == 0) record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                break;
            }
            if (meta[s].tile < 0) break;
            if (!mbar_wait_warp(&full_pay[s], u & 1u, p.timeout_ns, lane)) {
                if (lane == 0) record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                break;
            }
            const uint64_t prefix = meta[s].prefix;
            const bool write = prefix != POISON;
            const uint64_t gpos = prefix + meta[s].warp_base[cw];
            const uint32_t a = static_cast<uint32_t>(gpos % VEC);
            uint32_t run = a;
            if (write) {
                const T* seg = reinterpret_cast<const T*>(pay + s * TILE_BYTES) + cw * E;
                const uint32_t* segm = msk + s * W + cw * SW;
#pragma unroll
                for (uint32_t pass = 0; pass < PASSES; ++pass) {
                    const uint32_t m = (lane < WPP) ? segm[pass * WPP + lane] : 0u;
                    const uint32_t c = __popc(m);
                    const uint32_t incl = warp_incl_scan(c, lane);
                    const uint32_t excl = incl - c;
                    const uint32_t pass_total = __shfl_sync(0xffffffffu, incl, 31);
#pragma unroll
                    for (uint32_t g = 0; g < GROUPS; ++g) {
                        const uint32_t src = g * VEC + lane / (32 / VEC);
                        const uint32_t mw = __shfl_sync(0xffffffffu, m, src);
                        const uint32_t me = __shfl_sync(0xffffffffu, excl, src);
                        const uint32_t sh = (lane * VEC) & 31u;
                        const uint32_t bits = (mw >> sh) & ((1u << VEC) - 1u);
                        if (bits) {
                            uint32_t pos = run + me + __popc(mw & ((1u << sh) - 1u));
                            union {
                                uint4 v;
                                T e[VEC];
                            } x;
                            x.v = lds128(seg + pass * WPP * 32 + g * 32 * VEC + lane * VEC);
#pragma unroll
                            for (uint32_t e = 0; e < VEC; ++e)
                                if ((bits >> e) & 1u) stage[pos++] = x.e[e];
                        }
                    }
                    run += pass_total;
                }
            }
            __syncwarp();
            mbar_arrive(&empty[s]); // this warp no longer reads stage s
            if (write) {
                const uint32_t nvec = (run + VEC - 1) / VEC;
                uint8_t* gdst = p.out + (gpos - a) * sizeof(T);
                for (uint32_t v = lane; v < nvec; v += 32) {
                    const uint32_t e0 = v * VEC;
                    const uint32_t e1 = e0 + VEC;
                    if (e0 >= a && e1 <= run) {
                        stg128_cs(gdst + v * 16u, lds128(stage + e0));
                    } else {
                        const uint32_t lo = e0 > a ? e0 : a;
                        const uint32_t hi = e1 < run ? e1 : run;
                        for (uint32_t e = lo; e < hi; ++e) reinterpret_cast<T*>(gdst)[e] = stage[e];
                    }
                }
            }
            __syncwarp();
        }
    }

    if (MODE == 0) lookback_kernel_epilogue(p.hdr, &p.hdr->tile_counter, &p.hdr->done_counter, &s_flag, false, 0, 0);
}

// ---------------------------------------------------------------------------------
// Host side: per-device attribute setup and dispatch.
// ---------------------------------------------------------------------------------
size_t compact_tma_smem_bytes(uint32_t elem_bytes)
{
    switch (elem_bytes) {
        case 1: return Layout<uint8_t, STAGES, NCW>::TOTAL;
        case 2: return Layout<uint16_t, STAGES, NCW>::TOTAL;
        case 4: return Layout<uint32_t, STAGES, NCW>::TOTAL;
        case 8: return Layout<uint64_t, STAGES, NCW>::TOTAL;
        default: return 0;
    }
}

namespace {
constexpr int MAX_DEVICES = 64;
// bit (wi*2 + mode) set once the smem attribute was applied on that device
unsigned g_attr_done[MAX_DEVICES];

template <typename T, int MODE>
cudaError_t ensure_attr(int dev)
{
    constexpr int wi = (sizeof(T) == 1) ? 0 : (sizeof(T) == 2) ? 1 : (sizeof(T) == 4) ? 2 : 3;
    const unsigned bit = 1u << (wi * 2 + MODE);
    if (dev >= 0 && dev < MAX_DEVICES && (__atomic_load_n(&g_attr_done[dev], __ATOMIC_ACQUIRE) & bit)) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_compact_tma<T, MODE, STAGES, NCW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(Layout<T, STAGES, NCW>::TOTAL));
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < MAX_DEVICES) __atomic_fetch_or(&g_attr_done[dev], bit, __ATOMIC_RELEASE);
    return cudaSuccess;
}

template <typename T, int MODE>
cudaError_t launch_t(const CompactParams& p, uint32_t grid, cudaStream_t stream)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = ensure_attr<T, MODE>(dev);
    if (e != cudaSuccess) return e;
    k_compact_tma<T, MODE, STAGES, NCW><<<grid, NTHREADS, Layout<T, STAGES, NCW>::TOTAL, stream>>>(p);
    note_launch();
    return cudaGetLastError();
}

template <typename T, int MODE>
int blocks_per_sm_t()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (ensure_attr<T, MODE>(dev) != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_compact_tma<T, MODE, STAGES, NCW>, NTHREADS,
                                                      Layout<T, STAGES, NCW>::TOTAL) != cudaSuccess)
        return 0;
    return nb;
}
} // namespace

int compact_tma_blocks_per_sm(uint32_t elem_bytes, int mode)
{
    switch (elem_bytes) {
        case 1: return mode == 0 ? blocks_per_sm_t<uint8_t, 0>() : blocks_per_sm_t<uint8_t, 1>();
        case 2: return mode == 0 ? blocks_per_sm_t<uint16_t, 0>() : blocks_per_sm_t<uint16_t, 1>();
        case 4: return mode == 0 ? blocks_per_sm_t<uint32_t, 0>() : blocks_per_sm_t<uint32_t, 1>();
        case 8: return mode == 0 ? blocks_per_sm_t<uint64_t, 0>() : blocks_per_sm_t<uint64_t, 1>();
        default: return 0;
    }
}

cudaError_t launch_compact_tma(const CompactParams& p, uint32_t elem_bytes, int mode, uint32_t grid, cudaStream_t stream)
{
    switch (elem_bytes) {
        case 1: return mode == 0 ? launch_t<uint8_t, 0>(p, grid, stream) : launch_t<uint8_t, 1>(p, grid, stream);
        case 2: return mode == 0 ? launch_t<uint16_t, 0>(p, grid, stream) : launch_t<uint16_t, 1>(p, grid, stream);
        case 4: return mode == 0 ? launch_t<uint32_t, 0>(p, grid, stream) : launch_t<uint32_t, 1>(p, grid, stream);
        case 8: return mode == 0 ? launch_t<uint64_t, 0>(p, grid, stream) : launch_t<uint64_t, 1>(p, grid, stream);
        default: return cudaErrorInvalidValue;
    }
}

} // namespace cs
