// cs_kernels.cu — chunk popcount (pass 1), single-pass look-back scan (pass 2),
// warp-per-word writeout (the alignment-agnostic pass 3), workspace init and the seeded
// input generators.
#include <atomic>
#include <cstdint>
#include <cuda_runtime.h>

#include "cs_internal.cuh"

namespace cs {

// ---------------------------------------------------------------------------------
// Pass 1: per-chunk popcount.
// Reference: kernel_3pass_popc_none_striding (src/kernels/kernel_3pass.cuh:12-38) assigns
// one thread per chunk and walks it with strided 4-byte loads. Here consecutive threads
// read consecutive mask words (fully coalesced) and chunks are reduced with shuffles:
// chunks of <= 32 words are segmented warp reductions, longer chunks are warp-strided.
// Bits at positions >= n are masked off, so the mask tail need not be zero.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t load_mask_word(const uint32_t* mask, uint64_t wi, uint64_t nw, uint64_t n)
{
    if (wi >= nw) return 0u;
    uint32_t m = __ldg(mask + wi);
    if (wi == nw - 1 && (n & 31u)) m &= (1u << (n & 31u)) - 1u;
    return m;
}

// Vector form (16-byte-aligned mask, 128 <= L <= 4096): a warp step reads 32 uint4 (128 words
// = 4096 elements) and four steps are unrolled so four loads per lane are in flight; chunks
// of LPC = L/128 lanes are reduced with xor shuffles. Each unrolled warp iteration covers an
// aligned block of 16384 elements; when `hdr` is given, each CTA records in cta_flags whether
// one of its blocks holds at most 16384/32 selected elements, and the scan that follows
// turns that into hdr->sparse_epoch so the hybrid writeout knows to look for sparse units.
template <int LPC>
__global__ void __launch_bounds__(256) k_popc_chunks_vec(const uint32_t* __restrict__ mask, uint64_t n,
                                                         uint32_t* __restrict__ counts, ws_header* hdr,
                                                         uint32_t* __restrict__ cta_flags)
{
    __shared__ uint32_t s_sparse;
    if (threadIdx.x == 0) s_sparse = 0;
    __syncthreads();
    constexpr int UNROLL = 4;
    const uint64_t nw = (n + 31) / 32;
    const uint64_t nvec = (nw + 3) / 4;
    const uint64_t num_chunks = (nw + 4 * LPC - 1) / (4 * LPC);
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp_global = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t total_warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    const uint4* mv = reinterpret_cast<const uint4*>(mask);
    bool sparse_block = false;
    for (uint64_t base = warp_global * 32 * UNROLL; base < nvec; base += total_warps * 32 * UNROLL) {
        uint4 q[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            const uint64_t v = base + u * 32 + lane;
            if (v * 4 + 3 < nw) {
                q[u] = __ldg(mv + v);
                if (v * 4 + 3 == nw - 1 && (n & 31u)) q[u].w &= (1u << (n & 31u)) - 1u;
            } else {
                q[u].x = load_mask_word(mask, v * 4 + 0, nw, n);
                q[u].y = load_mask_word(mask, v * 4 + 1, nw, n);
                q[u].z = load_mask_word(mask, v * 4 + 2, nw, n);
                q[u].w = load_mask_word(mask, v * 4 + 3, nw, n);
            }
        }
        uint32_t block = 0;
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            uint32_t c = __popc(q[u].x) + __popc(q[u].y) + __popc(q[u].z) + __popc(q[u].w);
            block += c;
#pragma unroll
            for (int d = LPC / 2; d > 0; d >>= 1) c += __shfl_xor_sync(0xffffffffu, c, d);
            const uint64_t chunk = (base + u * 32 + lane) / LPC;
            if ((lane % LPC) == 0 && chunk < num_chunks) counts[chunk] = c;
        }
        if (hdr) {
            block = warp_sum32(block);
            sparse_block |= block <= (16384u / 32u);
        }
    }
    // one flag word per CTA (distinct addresses: same-address stores from every warp would
    // serialise in L2); the scan's last CTA folds them into hdr->sparse_epoch
    if (hdr) {
        if (lane == 0 && sparse_block) s_sparse = 1u;
        __syncthreads();
        if (threadIdx.x == 0) {
            if (blockIdx.x == 0) hdr->popc_ctas = gridDim.x;
            cta_flags[blockIdx.x] = s_sparse ? hdr->epoch : 0u;
        }
    }
}

// Scalar form (any 4-byte-aligned mask, any chunk length). It never proves the absence of
// sparse blocks, so with `hdr` it always flags the call.
__global__ void __launch_bounds__(256) k_popc_chunks(const uint32_t* __restrict__ mask, uint64_t n, uint32_t chunk_log2,
                                                     uint32_t* __restrict__ counts, ws_header* hdr,
                                                     uint32_t* __restrict__ cta_flags)
{
    const uint64_t nw = (n + 31) / 32;
    const uint32_t wpc_log2 = chunk_log2 - 5; // words per chunk = 2^wpc_log2
    const uint64_t num_chunks = (n + (1ull << chunk_log2) - 1) >> chunk_log2;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp_global = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t total_warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    if (hdr && blockIdx.x == 0 && threadIdx.x == 0) {
        hdr->popc_ctas = 1;
        cta_flags[0] = hdr->epoch;
    }
    if (wpc_log2 <= 5) {
        const uint32_t wpc = 1u << wpc_log2;
        const uint64_t nw_round = (nw + 31) & ~31ull;
        for (uint64_t base = warp_global * 32; base < nw_round; base += total_warps * 32) {
            const uint64_t wi = base + lane;
            uint32_t c = __popc(load_mask_word(mask, wi, nw, n));
            for (uint32_t off = wpc >> 1; off > 0; off >>= 1) c += __shfl_down_sync(0xffffffffu, c, off);
            if ((lane & (wpc - 1)) == 0) {
                const uint64_t chunk = wi >> wpc_log2;
                if (chunk < num_chunks) counts[chunk] = c;
            }
        }
    } else {
        const uint64_t wpc = 1ull << wpc_log2;
        for (uint64_t chunk = warp_global; chunk < num_chunks; chunk += total_warps) {
            uint32_t c = 0;
            const uint64_t w0 = chunk * wpc;
            for (uint64_t wi = w0 + lane; wi < w0 + wpc; wi += 32) c += __popc(load_mask_word(mask, wi, nw, n));
            c = warp_sum32(c);
            if (lane == 0) counts[chunk] = c;
        }
    }
}

cudaError_t launch_popc_chunks(const uint32_t* mask, uint64_t n, uint32_t chunk_log2, uint32_t* counts, ws_header* hdr,
                               uint32_t* cta_flags, int num_sms, cudaStream_t stream)
{
    const uint64_t nw = (n + 31) / 32;
    const bool vec = (reinterpret_cast<uintptr_t>(mask) & 15u) == 0 && chunk_log2 >= 7 && chunk_log2 <= 12;
    if (vec) {
        uint64_t blocks = ((nw + 3) / 4 + 1023) / 1024; // 8 warps x 128 vectors per block iteration
        uint64_t cap = static_cast<uint64_t>(num_sms) * 8;
        if (cap > POPC_FLAG_SLOTS) cap = POPC_FLAG_SLOTS;
        if (blocks > cap) blocks = cap;
        if (blocks == 0) blocks = 1;
        const unsigned g = static_cast<unsigned>(blocks);
        switch (chunk_log2) {
            case 7: k_popc_chunks_vec<1><<<g, 256, 0, stream>>>(mask, n, counts, hdr, cta_flags); break;
            case 8: k_popc_chunks_vec<2><<<g, 256, 0, stream>>>(mask, n, counts, hdr, cta_flags); break;
            case 9: k_popc_chunks_vec<4><<<g, 256, 0, stream>>>(mask, n, counts, hdr, cta_flags); break;
            case 10: k_popc_chunks_vec<8><<<g, 256, 0, stream>>>(mask, n, counts, hdr, cta_flags); break;
            case 11: k_popc_chunks_vec<16><<<g, 256, 0, stream>>>(mask, n, counts, hdr, cta_flags); break;
            default: k_popc_chunks_vec<32><<<g, 256, 0, stream>>>(mask, n, counts, hdr, cta_flags); break;
        }
    } else {
        uint64_t blocks = (nw + 255) / 256;
        const uint64_t cap = static_cast<uint64_t>(num_sms) * 8;
        if (blocks > cap) blocks = cap;
        if (blocks == 0) blocks = 1;
        k_popc_chunks<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(mask, n, chunk_log2, counts, hdr,
                                                                          cta_flags);
    }
    note_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// Pass 2: exclusive prefix sum of chunk counts, single pass with decoupled look-back.
// Reference: the hand-written up-sweep tree (kernel_3pass_pss_gmem_*, log2(C) launches,
// src/kernels/kernel_3pass.cuh:69-153) plus d_3pass_pproc_pssidx (:155-185), and the CUB
// ExclusiveSum it was replaced by (src/cub_wraps.cuh:52-79). Tiles of 4096 counts are
// taken in order from a device counter, so a tile only ever waits on tiles already held
// by running CTAs. The last tile writes the grand total (the selected count).
// ---------------------------------------------------------------------------------
__global__ void __launch_bounds__(SCAN_THREADS) k_scan(ScanParams p)
{
    __shared__ uint64_t s_warp[SCAN_THREADS / 32];
    __shared__ uint64_t s_tile_total;
    __shared__ uint32_t s_tile;
    __shared__ uint32_t s_flag;
    __shared__ LookbackSmem<SCAN_THREADS / 32> s_lb;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    const uint32_t epoch = p.hdr->epoch;

    while (true) {
        if (tid == 0) s_tile = atomicAdd(&p.hdr->scan_tile_counter, 1u);
        __syncthreads();
        const uint64_t tile = s_tile;
        if (tile >= p.num_tiles) break;
        const uint64_t base = tile * SCAN_TILE + static_cast<uint64_t>(tid) * SCAN_ITEMS_PER_THREAD;
        uint32_t v[SCAN_ITEMS_PER_THREAD];
        if (base + SCAN_ITEMS_PER_THREAD <= p.count && (reinterpret_cast<uintptr_t>(p.counts) & 15u) == 0) {
            const uint4* q = reinterpret_cast<const uint4*>(p.counts + base);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const uint4 x = __ldg(q + i);
                v[4 * i + 0] = x.x;
                v[4 * i + 1] = x.y;
                v[4 * i + 2] = x.z;
                v[4 * i + 3] = x.w;
            }
        } else {
#pragma unroll
            for (int i = 0; i < (int)SCAN_ITEMS_PER_THREAD; ++i) v[i] = (base + i < p.count) ? __ldg(p.counts + base + i) : 0u;
        }
        uint64_t thread_total = 0;
#pragma unroll
        for (int i = 0; i < (int)SCAN_ITEMS_PER_THREAD; ++i) thread_total += v[i];
        const uint64_t incl = warp_incl_scan64(thread_total, lane);
        if (lane == 31) s_warp[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            const uint64_t wt = lane < SCAN_THREADS / 32 ? s_warp[lane] : 0ull;
            const uint64_t wincl = warp_incl_scan64(wt, lane);
            const uint64_t tile_total = __shfl_sync(0xffffffffu, wincl, SCAN_THREADS / 32 - 1);
            if (lane < SCAN_THREADS / 32) s_warp[lane] = wincl - wt;
            if (lane == 0) s_tile_total = tile_total;
        }
        __syncthreads();
        const uint64_t prefix =
            lookback_cta<SCAN_THREADS>(p.status, tile, s_tile_total, epoch, p.timeout_ns, p.hdr, s_lb);
        if (prefix == POISON) {
#pragma unroll
            for (int i = 0; i < (int)SCAN_ITEMS_PER_THREAD; ++i)
                if (base + i < p.count) p.offsets[base + i] = POISON;
            if (tile == p.num_tiles - 1 && tid == 0 && p.total) *p.total = POISON;
        } else {
            uint64_t run = prefix + s_warp[warp] + (incl - thread_total);
#pragma unroll
            for (int i = 0; i < (int)SCAN_ITEMS_PER_THREAD; ++i) {
                if (base + i < p.count) p.offsets[base + i] = run;
                run += v[i];
            }
            if (tile == p.num_tiles - 1 && tid == 0 && p.total) *p.total = prefix + s_tile_total;
        }
        __syncthreads();
    }
    lookback_kernel_epilogue(p.hdr, &p.hdr->scan_tile_counter, &p.hdr->scan_done_counter, &s_flag, true, p.keep_begin,
                             p.keep_end, p.popc_flags);
}

cudaError_t launch_scan(const ScanParams& p, int num_sms, cudaStream_t stream)
{
    uint64_t blocks = p.num_tiles;
    const uint64_t cap = static_cast<uint64_t>(num_sms) * 4;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    k_scan<<<static_cast<unsigned>(blocks), SCAN_THREADS, 0, stream>>>(p);
    note_launch();
    return cudaGetLastError();
}


// Pass 1 of the hybrid writeout: the units of block `bl` of a column (UE = 131072 / w
// elements = 32 / w rows of 4096, always whole inside a 2^18-element block) whose count is
// at most UE / 32 belong to the sparse gather: their 16K-element items get this call's
// epoch in p.item_flags, and the gather visits only items so marked (a flag left by a call
// one epoch cycle ago costs the gather one test of the offsets, never a wrong write).
// s_warp / s_whalf: selected elements in each warp's 8 rows and in their first 4 rows.
// Called by all threads after those are written.
__device__ __forceinline__ void mark_sparse_units(const BlockScanParams& p, const ColumnDesc& col, uint64_t bl,
                                                  const uint32_t* s_warp, const uint32_t* s_whalf, uint32_t epoch)
{
    const uint32_t w = col.elem_bytes;
    const uint32_t rpu = 32u / w;     // rows per unit
    const uint32_t units = 64u / rpu; // units per block
    const uint32_t t = threadIdx.x;
    if (t >= units) return;
    uint32_t cnt;
    if (w == 8) cnt = (t & 1u) ? s_warp[t >> 1] - s_whalf[t >> 1] : s_whalf[t >> 1];
    else if (w == 4) cnt = s_warp[t];
    else if (w == 2) cnt = s_warp[2 * t] + s_warp[2 * t + 1];
    else cnt = s_warp[4 * t] + s_warp[4 * t + 1] + s_warp[4 * t + 2] + s_warp[4 * t + 3];
    const uint64_t ue = 131072u / w;
    const uint64_t e0 = (bl << SCAN_BLOCK_LOG2) + static_cast<uint64_t>(t) * ue;
    if (e0 >= col.n || cnt > ue / 32) return;
    const uint64_t e1 = e0 + ue < col.n ? e0 + ue : col.n;
    for (uint64_t it = e0 / 16384; it < (e1 + 16383) / 16384; ++it) p.item_flags[col.item_base + it] = epoch;
}

// ---------------------------------------------------------------------------------
// Pass 1 + 2 as one reduce-then-scan kernel (3-pass form, chunk length L = 128 .. 4096,
// 16-byte-aligned masks). A column is cut into blocks of 2^18 elements (32 KB of mask). A
// CTA takes whole blocks by static assignment and never waits on another CTA: its 8 warps
// each load 8 rows of 32 uint4 (4096 elements per row) in one round, each lane's share of a
// chunk is summed over the LPC = L/128 lanes holding the chunk, and warp and block scans
// give every chunk its offset within the block; the block's sum goes to blk_sum. The last
// CTA to finish scans the block sums into blk_base (exclusive prefix of each block within
// its column) and writes every column's count; consumers add the two (chunk_offset). This
// replaces a decoupled look-back across blocks, whose waiting dominated the fused pass at
// large n. Each CTA also records whether one of its aligned 16K-element groups holds at
// most 512 selected elements (the sparse-unit hint of the hybrid writeout).
// Reference: pass 1 kernel_3pass_popc_none_striding (src/kernels/kernel_3pass.cuh:12-57)
// and pass 2 launch_cub_pss / kernel_3pass_pss_gmem (src/cub_wraps.cuh:52-79,
// src/kernels/kernel_3pass.cuh:59-214).
// ---------------------------------------------------------------------------------

// This warp's 8 rows (32 uint4 each) of block `bl` of `col`, read from global memory: the
// last word of the column has its bits past n cleared, and words past the column read 0.
__device__ __forceinline__ void popc_block_load(const ColumnDesc& col, uint64_t bl, uint32_t warp, uint32_t lane,
                                                uint4 (&q)[8])
{
    const uint64_t n = col.n;
    const uint64_t nw = (n + 31) / 32;
    const uint32_t* __restrict__ mask = col.mask;
    const uint4* mv = reinterpret_cast<const uint4*>(mask);
    const uint64_t row0 = bl * 64 + warp * 8; // this warp's first row (4096 elements each)
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const uint64_t vi = (row0 + r) * 32 + lane;
        if (vi * 4 + 3 < nw) {
            q[r] = __ldg(mv + vi);
            if (vi * 4 + 3 == nw - 1 && (n & 31u)) q[r].w &= (1u << (n & 31u)) - 1u;
        } else {
            uint32_t w4[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint64_t wi = vi * 4 + k;
                w4[k] = 0;
                if (wi < nw) {
                    w4[k] = __ldg(mask + wi);
                    if (wi == nw - 1 && (n & 31u)) w4[k] &= (1u << (n & 31u)) - 1u;
                }
            }
            q[r] = make_uint4(w4[0], w4[1], w4[2], w4[3]);
        }
    }
}

// The rest of a block once every warp holds its rows in q: chunk offsets within the block,
// the block sum, the sparse hint (sparse_seen) and, in the hybrid form, the sparse-unit
// marks. Called by all 256 threads; returns after a barrier, so s_warp may be rewritten.
// s_epoch (written by thread 0 before its first call) is read after the first barrier here.
template <int LPC>
__device__ __forceinline__ void popc_block_finish(const BlockScanParams& p, const ColumnDesc& col, uint64_t blk,
                                                  uint64_t bl, const uint4 (&q)[8], uint32_t* s_warp,
                                                  uint32_t* s_whalf, const uint32_t* s_epoch, bool& sparse_seen)
{
    constexpr uint32_t CHUNK_LOG2 = LPC == 1 ? 7 : LPC == 2 ? 8 : LPC == 4 ? 9 : LPC == 8 ? 10 : LPC == 16 ? 11 : 12;
    static_assert((1u << CHUNK_LOG2) == LPC * 128u, "chunk length = 128 elements per lane");
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    const uint64_t n = col.n;
    const uint64_t nchunks = (n + (1ull << CHUNK_LOG2) - 1) >> CHUNK_LOG2;
    const uint64_t row0 = bl * 64 + warp * 8;
    uint32_t rel[8]; // offset of this lane's chunk within the warp's 8 rows
    uint32_t run = 0, half = 0;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const uint32_t c = __popc(q[r].x) + __popc(q[r].y) + __popc(q[r].z) + __popc(q[r].w);
        if constexpr (LPC == 32) {
            // a chunk is a whole row: its offset is the run before it, its count one reduction
            rel[r] = run;
            run += __reduce_add_sync(0xffffffffu, c);
            if (r == 3) half = run;
            continue;
        }
        const uint32_t incl = warp_incl_scan(c, lane);
        // the chunk's in-row offset: the exclusive scan at its first lane
        const uint32_t ex = __shfl_sync(0xffffffffu, incl - c, lane & ~static_cast<uint32_t>(LPC - 1));
        rel[r] = run + ex;
        run += __shfl_sync(0xffffffffu, incl, 31);
        if (r == 3) half = run;
    }
    // sparse hint over the warp's two aligned 16K-element groups (rows 0-3, 4-7)
    sparse_seen |= (half <= 512u) && row0 * 4096 < n;
    sparse_seen |= (run - half <= 512u) && (row0 + 4) * 4096 < n;
    if (lane == 0) {
        s_warp[warp] = run;
        s_whalf[warp] = half;
    }
    __syncthreads();
    if (p.item_flags) mark_sparse_units(p, col, bl, s_warp, s_whalf, *s_epoch);
    uint32_t wbase = 0, btot = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) {
        const uint32_t v = s_warp[w];
        wbase += (static_cast<uint32_t>(w) < warp) ? v : 0u;
        btot += v;
    }
    if ((lane & static_cast<uint32_t>(LPC - 1)) == 0u) {
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const uint64_t chunk = ((row0 + r) * 32 + lane) / LPC;
            if (chunk < nchunks) col.offsets[chunk] = wbase + rel[r];
        }
    }
    if (tid == 0) p.blk_sum[blk] = btot;
    __syncthreads(); // s_warp is rewritten by the next block
}

// The end of both pass-1+2 kernels (all threads): the finishing ticket carries the CTA's
// sparse hint in its upper bits, so the last CTA learns from its own atomic whether any CTA
// saw a sparse block (no flag array to read). The last CTA scans the block sums and closes
// the epoch; the call's scan is marked clean unless a CTA poisoned this epoch.
__device__ __forceinline__ void popc_blocks_finish_grid(const BlockScanParams& p, bool sparse_seen,
                                                        const uint32_t* s_epoch, uint32_t* s_flag, uint64_t* s_scan)
{
    const uint32_t tid = threadIdx.x;
    const bool cta_sparse = __syncthreads_or(sparse_seen) != 0;
    const uint32_t epoch = *s_epoch; // written by thread 0 before the barrier above
    if (tid == 0) {
        __threadfence(); // this CTA's offsets and block sums before its ticket
        const uint32_t prev = atomicAdd(&p.hdr->scan_done_counter, 1u + (cta_sparse ? 0x10000u : 0u));
        const bool last = (prev & 0xffffu) == gridDim.x - 1;
        *s_flag = last ? (1u | ((cta_sparse || (prev >> 16) != 0u) ? 2u : 0u)) : 0u;
    }
    __syncthreads();
    const uint32_t fin = *s_flag;
    if (!(fin & 1u)) return;
    __threadfence(); // every other CTA's block sums (and any poison mark) are visible
    const bool clean = reinterpret_cast<volatile ws_header*>(p.hdr)->poison_epoch != epoch;
    blocks_last_cta(p, s_scan, clean);
    epilogue_last_blocks(p.hdr, epoch, (fin & 2u) != 0u, p.keep_begin, p.keep_end, clean);
}

template <int LPC>
__global__ void __launch_bounds__(256, 4) k_popc_blocks(const BlockScanParams p)
{
    __shared__ uint32_t s_warp[8];
    __shared__ uint32_t s_whalf[8];
    __shared__ uint64_t s_scan[8];
    __shared__ uint32_t s_flag;
    __shared__ uint32_t s_epoch;
    const uint32_t tid = threadIdx.x;
    grid_dependency_wait(); // earlier calls may still be using this workspace
    if (tid == 0) s_epoch = p.hdr->epoch;
    bool sparse_seen = false;
    for (uint64_t blk = blockIdx.x; blk < p.num_blocks; blk += gridDim.x) {
        const ColumnDesc& col = column_of(p.col0, p.cols, p.blk_col, blk);
        const uint64_t bl = blk - col.tile_base; // block within its column
        uint4 q[8];
        popc_block_load(col, bl, tid >> 5, tid & 31u, q);
        popc_block_finish<LPC>(p, col, blk, bl, q, s_warp, s_whalf, &s_epoch, sparse_seen);
    }
    popc_blocks_finish_grid(p, sparse_seen, &s_epoch, &s_flag, s_scan);
}

// ---------------------------------------------------------------------------------
// Pass 1 + 2, streaming form for long masks (more than 4 blocks per SM, where the
// register-staged k_popc_blocks needs a second round of CTAs and pays the load latency and
// the tail of a round twice). POPC_STREAM_CTAS CTAs per SM each take a contiguous range of
// blocks; thread 0 streams them through POPC_STAGES shared-memory stages of 32 KB with 1-D
// bulk copies (cp.async.bulk, no multicast), so the next block of every CTA is in flight
// while its warps count the current one. A stage is refilled once every warp has left the
// block it held (the barrier that ends popc_block_finish). A block that is not whole (the
// last block of a column whose length is not a multiple of 2^18) is read from global memory
// as in k_popc_blocks. The per-block work and the end are those of k_popc_blocks.
// The shape was measured on B200 at 2^28 f32 and 2^29 u8/u16 (3-pass calls, us per call):
// 3 CTAs x 2 stages beat 1 x 6 (the counting of one CTA's 8 warps is latency-bound, so one
// CTA per SM left the copies waiting on it), 2 x 3 and 4 x 1.
// A stage wait that runs out records DEVERR_PIPELINE_TIMEOUT and poisons the call's scan;
// the CTA then issues no further copies and waits (bounded) for the ones in flight.
// ---------------------------------------------------------------------------------
#ifndef CS_POPC_STAGES
#define CS_POPC_STAGES 2
#endif
#ifndef CS_POPC_STREAM_CTAS
#define CS_POPC_STREAM_CTAS 3
#endif
constexpr uint32_t POPC_STAGES = CS_POPC_STAGES;
constexpr int POPC_STREAM_CTAS = CS_POPC_STREAM_CTAS; // CTAs per SM
constexpr uint32_t MASK_BLOCK_BYTES = (1u << SCAN_BLOCK_LOG2) / 8; // 32 KB of mask per block
constexpr uint64_t POPC_WAIT_NS = 2000000000ull; // bound on one stage wait (a copy lands in microseconds)
constexpr uint32_t POPC_STREAM_SMEM = POPC_STAGES * MASK_BLOCK_BYTES;

template <int LPC>
__global__ void __launch_bounds__(256, POPC_STREAM_CTAS) k_popc_stream(const BlockScanParams p)
{
    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ __align__(8) uint64_t s_full[POPC_STAGES];
    __shared__ uint32_t s_warp[8];
    __shared__ uint32_t s_whalf[8];
    __shared__ uint64_t s_scan[8];
    __shared__ uint32_t s_flag;
    __shared__ uint32_t s_epoch;
    __shared__ uint32_t s_fail;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    const uint64_t b0 = blockIdx.x * p.num_blocks / gridDim.x;
    const uint64_t b1 = (blockIdx.x + 1ull) * p.num_blocks / gridDim.x;
    if (tid == 0) {
        for (uint32_t s = 0; s < POPC_STAGES; ++s) mbar_init(&s_full[s], 1);
        fence_mbar_init();
        s_fail = 0u;
    }
    grid_dependency_wait(); // the mask may come from the previous kernel, the workspace too
    // a block is copied in bulk when all its bits lie inside its column
    auto whole = [&](const ColumnDesc& c, uint64_t bl) -> bool { return ((bl + 1) << SCAN_BLOCK_LOG2) <= c.n; };
    uint32_t pending = 0; // thread 0: stages with a copy in flight
    auto issue = [&](uint64_t blk, uint32_t s) {
        const ColumnDesc& c = column_of(p.col0, p.cols, p.blk_col, blk);
        const uint64_t bl = blk - c.tile_base;
        if (!whole(c, bl)) return;
        mbar_arrive_expect_tx(&s_full[s], MASK_BLOCK_BYTES);
        bulk_g2s(smem + s * MASK_BLOCK_BYTES, c.mask + bl * (MASK_BLOCK_BYTES / 4), MASK_BLOCK_BYTES, &s_full[s]);
        pending |= 1u << s;
    };
    if (tid == 0) {
        // the first copies go out before the header read (thread 0 initialised the barriers)
        for (uint32_t k = 0; k < POPC_STAGES && b0 + k < b1; ++k) issue(b0 + k, k);
        s_epoch = p.hdr->epoch;
    }
    __syncthreads(); // barriers initialised, s_epoch and s_fail visible
    const uint32_t epoch = s_epoch;
    bool sparse_seen = false;
    uint32_t parity = 0; // bit s: parity of the phase stage s completes next
    for (uint64_t i = 0; b0 + i < b1; ++i) {
        const uint64_t blk = b0 + i;
        const uint32_t s = static_cast<uint32_t>(i % POPC_STAGES);
        const ColumnDesc& col = column_of(p.col0, p.cols, p.blk_col, blk);
        const uint64_t bl = blk - col.tile_base;
        uint4 q[8];
        if (whole(col, bl)) {
            // after a failure no stage is refilled, so nothing more is waited for
            if (*reinterpret_cast<volatile uint32_t*>(&s_fail) == 0u) {
                if (mbar_wait_bounded(&s_full[s], (parity >> s) & 1u, POPC_WAIT_NS)) {
                    parity ^= 1u << s;
                    if (tid == 0) pending &= ~(1u << s);
                } else {
                    atomicOr(&s_fail, 1u);
                    if (lane == 0) {
                        record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                        reinterpret_cast<volatile ws_header*>(p.hdr)->poison_epoch = epoch;
                    }
                }
            }
            const uint4* sv = reinterpret_cast<const uint4*>(smem + s * MASK_BLOCK_BYTES);
#pragma unroll
            for (int r = 0; r < 8; ++r) q[r] = sv[(warp * 8 + r) * 32 + lane];
        } else {
            popc_block_load(col, bl, warp, lane, q);
        }
        popc_block_finish<LPC>(p, col, blk, bl, q, s_warp, s_whalf, &s_epoch, sparse_seen);
        // every warp has left stage s (the barrier ending popc_block_finish): refill it
        if (tid == 0 && b0 + i + POPC_STAGES < b1 && s_fail == 0u) issue(b0 + i + POPC_STAGES, s);
    }
    // after a failed wait: the copies still in flight (each stage's pending phase is the one
    // `parity` names) must land before the CTA exits
    if (tid == 0 && pending != 0u) {
        for (uint32_t s = 0; s < POPC_STAGES; ++s)
            if ((pending >> s) & 1u) mbar_wait_bounded(&s_full[s], (parity >> s) & 1u, POPC_WAIT_NS);
    }
    popc_blocks_finish_grid(p, sparse_seen, &s_epoch, &s_flag, s_scan);
}

// Masks of more than this many blocks per SM take the streaming form.
#ifndef CS_POPC_STREAM_BLOCKS_PER_SM
#define CS_POPC_STREAM_BLOCKS_PER_SM 4
#endif

namespace {
constexpr int POPC_MAX_DEVICES = 64;
unsigned g_popc_stream_attr[POPC_MAX_DEVICES]; // bit k: smem attribute of variant k applied

template <int LPC>
cudaError_t launch_popc_stream(const BlockScanParams& p, uint32_t grid, cudaStream_t stream, int variant)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned bit = 1u << variant;
    const bool known = dev >= 0 && dev < POPC_MAX_DEVICES;
    if (!known || !(__atomic_load_n(&g_popc_stream_attr[dev], __ATOMIC_ACQUIRE) & bit)) {
        e = cudaFuncSetAttribute(k_popc_stream<LPC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(POPC_STREAM_SMEM));
        if (e != cudaSuccess) return e;
        if (known) __atomic_fetch_or(&g_popc_stream_attr[dev], bit, __ATOMIC_RELEASE);
    }
    return launch_pdl(k_popc_stream<LPC>, dim3(grid), dim3(256), POPC_STREAM_SMEM, stream, p);
}
} // namespace

cudaError_t launch_popc_blocks(const BlockScanParams& p, int num_sms, cudaStream_t stream)
{
    cudaError_t e;
    if (num_sms > 0 && p.num_blocks > static_cast<uint64_t>(num_sms) * CS_POPC_STREAM_BLOCKS_PER_SM) {
        const uint32_t grid = static_cast<uint32_t>(num_sms) * POPC_STREAM_CTAS; // fewer CTAs than blocks
        switch (p.chunk_log2) {
            case 7: e = launch_popc_stream<1>(p, grid, stream, 0); break;
            case 8: e = launch_popc_stream<2>(p, grid, stream, 1); break;
            case 9: e = launch_popc_stream<4>(p, grid, stream, 2); break;
            case 10: e = launch_popc_stream<8>(p, grid, stream, 3); break;
            case 11: e = launch_popc_stream<16>(p, grid, stream, 4); break;
            case 12: e = launch_popc_stream<32>(p, grid, stream, 5); break;
            default: return cudaErrorInvalidValue;
        }
        note_launch();
        return e;
    }
    uint64_t blocks = p.num_blocks;
    uint64_t cap = static_cast<uint64_t>(num_sms) * 8;
    if (cap > POPC_FLAG_SLOTS) cap = POPC_FLAG_SLOTS;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    const dim3 g(static_cast<unsigned>(blocks)), b(256);
    switch (p.chunk_log2) {
        case 7: e = launch_pdl(k_popc_blocks<1>, g, b, 0, stream, p); break;
        case 8: e = launch_pdl(k_popc_blocks<2>, g, b, 0, stream, p); break;
        case 9: e = launch_pdl(k_popc_blocks<4>, g, b, 0, stream, p); break;
        case 10: e = launch_pdl(k_popc_blocks<8>, g, b, 0, stream, p); break;
        case 11: e = launch_pdl(k_popc_blocks<16>, g, b, 0, stream, p); break;
        case 12: e = launch_pdl(k_popc_blocks<32>, g, b, 0, stream, p); break;
        default: return cudaErrorInvalidValue;
    }
    note_launch();
    return e;
}

// ---------------------------------------------------------------------------------
// Pass 3, alignment-agnostic form: one warp per chunk walks the chunk's mask words; lane
// l owns element 32*w + l, its output slot is popc(word & lanemask_lt) past the running
// offset. Empty chunks are skipped using the pass-1 counts. Mirrors the reference's
// warp-cooperative writeout (kernel_3pass_proc_true_striding_naive_writeout,
// src/kernels/kernel_3pass.cuh:216-327) with LSB-first bits and 64-bit indexing.
// ---------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_writeout_naive(const T* __restrict__ in, const uint32_t* __restrict__ mask,
                                                        T* __restrict__ out, uint64_t n,
                                                        const uint64_t* __restrict__ chunk_offsets,
                                                        const uint32_t* __restrict__ chunk_counts, uint32_t chunk_log2,
                                                        const ws_header* hdr)
{
    __shared__ uint32_t s_hflags;
    if (!(cta_header_flags(hdr, &s_hflags) & 1u)) return; // pass 2 offsets not trustworthy: write nothing
    const uint64_t nw = (n + 31) / 32;
    const uint64_t num_chunks = (n + (1ull << chunk_log2) - 1) >> chunk_log2;
    const uint64_t wpc = 1ull << (chunk_log2 - 5);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt = (1u << lane) - 1u;
    const uint64_t warp_global = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t total_warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    for (uint64_t chunk = warp_global; chunk < num_chunks; chunk += total_warps) {
        if (chunk_counts && chunk_counts[chunk] == 0u) continue;
        uint64_t pos = chunk_offsets[chunk];
        if (pos == POISON) continue;
        const uint64_t w_end = (chunk + 1) * wpc < nw ? (chunk + 1) * wpc : nw;
        for (uint64_t wi = chunk * wpc; wi < w_end; ++wi) {
            const uint32_t m = load_mask_word(mask, wi, nw, n);
            if (m == 0u) continue;
            if ((m >> lane) & 1u) out[pos + __popc(m & lt)] = in[wi * 32 + lane];
            pos += __popc(m);
        }
    }
}

cudaError_t launch_writeout_naive(const void* in, const uint32_t* mask, void* out, uint64_t n, uint32_t elem_bytes,
                                  const uint64_t* chunk_offsets, const uint32_t* chunk_counts, uint32_t chunk_log2,
                                  const ws_header* hdr, int num_sms, cudaStream_t stream)
{
    const uint64_t num_chunks = (n + (1ull << chunk_log2) - 1) >> chunk_log2;
    uint64_t blocks = (num_chunks + 7) / 8;
    const uint64_t cap = static_cast<uint64_t>(num_sms) * 8;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    const unsigned g = static_cast<unsigned>(blocks);
    switch (elem_bytes) {
        case 1:
            k_writeout_naive<uint8_t><<<g, 256, 0, stream>>>(static_cast<const uint8_t*>(in), mask,
                                                             static_cast<uint8_t*>(out), n, chunk_offsets,
                                                             chunk_counts, chunk_log2, hdr);
            break;
        case 2:
            k_writeout_naive<uint16_t><<<g, 256, 0, stream>>>(static_cast<const uint16_t*>(in), mask,
                                                              static_cast<uint16_t*>(out), n, chunk_offsets,
                                                              chunk_counts, chunk_log2, hdr);
            break;
        case 4:
            k_writeout_naive<uint32_t><<<g, 256, 0, stream>>>(static_cast<const uint32_t*>(in), mask,
                                                              static_cast<uint32_t*>(out), n, chunk_offsets,
                                                              chunk_counts, chunk_log2, hdr);
            break;
        case 8:
            k_writeout_naive<uint64_t><<<g, 256, 0, stream>>>(static_cast<const uint64_t*>(in), mask,
                                                              static_cast<uint64_t*>(out), n, chunk_offsets,
                                                              chunk_counts, chunk_log2, hdr);
            break;
        default: return cudaErrorInvalidValue;
    }
    note_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// Pass 3, sparse units (3-pass hybrid, chunk length <= 4096). Units of the TMA kernel whose
// selected count is at most sparse_max are compacted here instead. A warp takes groups of 4
// blocks of 1024 elements (one mask word per lane per block), each starting on a chunk
// boundary, derives each block's output offset from the pass-2 chunk offset plus in-warp
// block popcounts, and lanes gather only their selected elements — DRAM traffic is the mask
// plus the sectors holding selected elements. The work is whole 16K-element items (4
// groups) when there are more items than resident warps, quarter items (one group) when
// there are fewer: a column with few sparse units then gets four times the warps, each with
// a quarter of the dependent steps (batch256 +3.5%, 2^24 u32 p = 0.01 40.0 -> 27.6 us), while
// many items keep the cheaper whole-item work (2^28 f32 p = 0.001: 56.6 us whole, 60.9
// quartered). A dense unit is rejected with two loads, and the whole kernel returns at once
// when pass 1 saw no sparse block. The TMA kernel skips exactly these units (same count test).
// ---------------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void sparse_groups(const ColumnDesc& c, uint64_t item, uint32_t g_begin, uint32_t g_end,
                                              uint32_t chunk_log2, uint32_t lane)
{
    const T* __restrict__ in = reinterpret_cast<const T*>(c.in);
    T* __restrict__ out = reinterpret_cast<T*>(c.out);
    const uint32_t* __restrict__ mask = c.mask;
    const uint64_t n = c.n;
    const uint64_t nw = (n + 31) / 32;
    const uint64_t nblocks = (n + 1023) / 1024;
    const uint64_t unit_elems = unit_elems_for(sizeof(T));
    const uint64_t sparse_max = unit_elems / 32;
    const uint64_t unit = (item * 16 * 1024) / unit_elems; // an item never straddles units
    const uint64_t u_end_elem = (unit + 1) * unit_elems;
    const uint64_t off_b = chunk_offset(c, (unit * unit_elems) >> chunk_log2, chunk_log2);
    const uint64_t off_e = u_end_elem >= n ? *c.d_count : chunk_offset(c, u_end_elem >> chunk_log2, chunk_log2);
    if (off_e - off_b > sparse_max) return; // dense unit: the TMA kernel owns it
    // groups of 4 blocks = 4096 elements start on chunk boundaries (chunk length <= 4096)
    for (uint64_t b0 = item * 16 + g_begin * 4; b0 < item * 16 + g_end * 4 && b0 < nblocks; b0 += 4) {
        uint32_t m[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint64_t wi = (b0 + k) * 32 + lane;
            m[k] = 0;
            if (wi < nw) {
                m[k] = __ldg(mask + wi);
                if (wi == nw - 1 && (n & 31u)) m[k] &= (1u << (n & 31u)) - 1u;
            }
        }
        uint64_t pos0 = chunk_offset(c, (b0 * 1024) >> chunk_log2, chunk_log2);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            // chunks shorter than a group: take the offset where a later chunk starts
            const uint64_t e0 = (b0 + k) * 1024;
            if (k > 0 && (e0 & ((1ull << chunk_log2) - 1)) == 0 && e0 < n) pos0 = chunk_offset(c, e0 >> chunk_log2, chunk_log2);
            const uint32_t cnt = __popc(m[k]);
            const uint32_t incl = warp_incl_scan(cnt, lane);
            if (__ballot_sync(0xffffffffu, m[k] != 0u) != 0u) {
                uint64_t pos = pos0 + incl - cnt;
                uint32_t mm = m[k];
                const uint64_t e_word = ((b0 + k) * 32 + lane) * 32;
                while (mm) {
                    const uint32_t b = __ffs(mm) - 1;
                    mm &= mm - 1;
                    out[pos++] = in[e_word + b];
                }
            }
            pos0 += __shfl_sync(0xffffffffu, incl, 31);
        }
    }
}

template <int SPLIT> // work items per 16K-element item: 1 (whole items) or 4 (quarters)
__global__ void __launch_bounds__(256) k_writeout_sparse(const SparseParams p)
{
    grid_dependency_wait(); // offsets and counts of pass 2
    __shared__ uint32_t s_hflags;
    const uint32_t hflags = cta_header_flags(p.hdr, &s_hflags);
    if (!(hflags & 1u)) return; // pass 2 offsets not trustworthy: write nothing
    if (!(hflags & 2u)) return; // no 16K block with <= 1/32 selected: no sparse unit
    // items pass 1 marked carry the epoch of that pass, the one before the current
    const uint32_t mark = p.item_flags ? prev_epoch(*reinterpret_cast<const volatile uint32_t*>(&p.hdr->epoch)) : 0u;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warp_global = (static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const uint64_t total_warps = (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5;
    // a warp tests 32 work items per round, taken round robin over all warps so that marked
    // items spread evenly whether few or all are marked
    static_assert(SPLIT == 1 || SPLIT == 4, "whole or quarter items");
    constexpr uint32_t gpw = 4u / SPLIT; // groups per work item
    const uint64_t num_work = p.num_items * SPLIT;
    for (uint64_t r0 = 0; warp_global + r0 * total_warps < num_work; r0 += 32) {
        const uint64_t mine = warp_global + (r0 + lane) * total_warps;
        const bool flagged = mine < num_work && (!p.item_flags || __ldg(p.item_flags + mine / SPLIT) == mark);
        uint32_t todo = __ballot_sync(0xffffffffu, flagged);
        while (todo) {
            const uint64_t work = warp_global + (r0 + (__ffs(todo) - 1)) * total_warps;
            todo &= todo - 1;
            const uint64_t item = work / SPLIT;
            const uint32_t g0 = static_cast<uint32_t>(work % SPLIT) * gpw;
            const ColumnDesc& c = column_of(p.col0, p.cols, p.item_col, item);
            const uint64_t il = item - c.item_base;
            switch (c.elem_bytes) {
                case 1: sparse_groups<uint8_t>(c, il, g0, g0 + gpw, p.chunk_log2, lane); break;
                case 2: sparse_groups<uint16_t>(c, il, g0, g0 + gpw, p.chunk_log2, lane); break;
                case 4: sparse_groups<uint32_t>(c, il, g0, g0 + gpw, p.chunk_log2, lane); break;
                default: sparse_groups<uint64_t>(c, il, g0, g0 + gpw, p.chunk_log2, lane); break;
            }
        }
    }
}

// CTAs of 256 threads of KERNEL resident on one SM at once (taken once). Grid-stride passes
// launch one wave of them: CTAs past the first wave would run their whole round-robin share
// after it.
template <auto KERNEL>
int resident_per_sm_256()
{
    static std::atomic<int> cached{0};
    int v = cached.load(std::memory_order_relaxed);
    if (v > 0) return v;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, KERNEL, 256, 0) != cudaSuccess || v < 1) {
        cudaGetLastError();
        v = 4;
    }
    cached.store(v, std::memory_order_relaxed);
    return v;
}

cudaError_t launch_writeout_sparse(const SparseParams& p, int num_sms, cudaStream_t stream)
{
    const bool quarters = p.num_items * 4 <= static_cast<uint64_t>(num_sms) * 64; // while there are warps for them
    const uint64_t per_sm = quarters ? resident_per_sm_256<k_writeout_sparse<4>>() : resident_per_sm_256<k_writeout_sparse<1>>();
    const uint64_t cap = static_cast<uint64_t>(num_sms) * per_sm; // CTAs of 8 warps
    uint64_t blocks = (p.num_items * (quarters ? 4 : 1) + 7) / 8;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    const cudaError_t e = quarters
        ? launch_pdl(k_writeout_sparse<4>, dim3(static_cast<unsigned>(blocks)), dim3(256), 0, stream, p)
        : launch_pdl(k_writeout_sparse<1>, dim3(static_cast<unsigned>(blocks)), dim3(256), 0, stream, p);
    note_launch();
    return e;
}

// ---------------------------------------------------------------------------------
// Workspace init: zero everything, then write the header.
// ---------------------------------------------------------------------------------
__global__ void k_ws_init(ws_header* hdr, uint64_t ws_bytes)
{
    uint4* p = reinterpret_cast<uint4*>(hdr);
    const uint64_t n16 = ws_bytes / 16u;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n16; i += stride)
        p[i] = make_uint4(0, 0, 0, 0);
}

__global__ void k_ws_header(ws_header* hdr, uint64_t ws_bytes)
{
    hdr->magic = WS_MAGIC;
    hdr->epoch = EPOCH_MIN;
    hdr->err = 0;
    hdr->tile_counter = 0;
    hdr->done_counter = 0;
    hdr->scan_tile_counter = 0;
    hdr->scan_done_counter = 0;
    hdr->ws_bytes = ws_bytes;
}

cudaError_t launch_ws_init(ws_header* hdr, size_t ws_bytes, cudaStream_t stream)
{
    uint64_t blocks = (ws_bytes / 16 + 255) / 256;
    if (blocks > 1024) blocks = 1024;
    if (blocks == 0) blocks = 1;
    k_ws_init<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(hdr, ws_bytes);
    k_ws_header<<<1, 1, 0, stream>>>(hdr, ws_bytes);
    note_launch(2);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------------
// Seeded generators. mix64 is the SplitMix64 output function (Steele, Lea, Flood 2014)
// applied to seed + (i+1)*golden-gamma, so element i depends only on (seed, i).
// ---------------------------------------------------------------------------------
__device__ __forceinline__ uint64_t mix64(uint64_t seed, uint64_t i)
{
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

template <typename T>
__global__ void k_gen_payload(T* out, uint64_t n, uint64_t seed, int float_unit)
{
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t h = mix64(seed, i);
        if (sizeof(T) == 4 && float_unit) {
            const float f = static_cast<float>(static_cast<uint32_t>(h >> 40)) * (1.0f / 16777216.0f);
            out[i] = static_cast<T>(__float_as_uint(f));
        } else {
            out[i] = static_cast<T>(h);
        }
    }
}

cudaError_t launch_gen_payload(void* out, uint64_t n, uint32_t elem_bytes, uint64_t seed, int float_unit, int num_sms,
                               cudaStream_t stream)
{
    uint64_t blocks = (n + 255) / 256;
    const uint64_t cap = static_cast<uint64_t>(num_sms) * 16;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    const unsigned g = static_cast<unsigned>(blocks);
    switch (elem_bytes) {
        case 1: k_gen_payload<uint8_t><<<g, 256, 0, stream>>>(static_cast<uint8_t*>(out), n, seed, 0); break;
        case 2: k_gen_payload<uint16_t><<<g, 256, 0, stream>>>(static_cast<uint16_t*>(out), n, seed, 0); break;
        case 4: k_gen_payload<uint32_t><<<g, 256, 0, stream>>>(static_cast<uint32_t*>(out), n, seed, float_unit); break;
        case 8: k_gen_payload<uint64_t><<<g, 256, 0, stream>>>(static_cast<uint64_t*>(out), n, seed, 0); break;
        default: return cudaErrorInvalidValue;
    }
    note_launch();
    return cudaGetLastError();
}

// word w packs elements 32w..32w+31, LSB-first; bit set iff (mix64(seed, i) >> 32) < threshold
__global__ void k_gen_mask_bernoulli(uint32_t* mask, uint64_t n, uint64_t threshold, uint64_t seed)
{
    const uint64_t nw = (n + 31) / 32;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t w = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w < nw; w += stride) {
        uint32_t m = 0;
        for (uint32_t b = 0; b < 32; ++b) {
            const uint64_t i = w * 32 + b;
            if (i < n && (mix64(seed, i) >> 32) < threshold) m |= 1u << b;
        }
        mask[w] = m;
    }
}

cudaError_t launch_gen_mask_bernoulli(uint32_t* mask, uint64_t n, uint64_t threshold, uint64_t seed, int num_sms,
                                      cudaStream_t stream)
{
    const uint64_t nw = (n + 31) / 32;
    uint64_t blocks = (nw + 255) / 256;
    const uint64_t cap = static_cast<uint64_t>(num_sms) * 16;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    k_gen_mask_bernoulli<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(mask, n, threshold, seed);
    note_launch();
    return cudaGetLastError();
}

// Alternating runs, step 1: toggle words (bit i set iff position i starts a new run),
// stored as their in-word prefix parity, plus per-word toggle popcounts for the scan.
__global__ void k_gen_runs_toggle(uint32_t* mask, uint32_t* parity_counts, uint64_t n, uint64_t threshold, uint64_t seed)
{
    const uint64_t nw = (n + 31) / 32;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t w = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w < nw; w += stride) {
        uint32_t t = 0;
        for (uint32_t b = 0; b < 32; ++b) {
            const uint64_t i = w * 32 + b;
            if (i < n && (mix64(seed, i) >> 32) < threshold) t |= 1u << b;
        }
        parity_counts[w] = static_cast<uint32_t>(__popc(t));
        uint32_t x = t; // bit j <- xor of bits 0..j
        x ^= x << 1;
        x ^= x << 2;
        x ^= x << 4;
        x ^= x << 8;
        x ^= x << 16;
        mask[w] = x;
    }
}

cudaError_t launch_gen_runs_toggle(uint32_t* mask, uint32_t* parity_counts, uint64_t n, uint64_t threshold,
                                   uint64_t seed, int num_sms, cudaStream_t stream)
{
    const uint64_t nw = (n + 31) / 32;
    uint64_t blocks = (nw + 255) / 256;
    const uint64_t cap = static_cast<uint64_t>(num_sms) * 16;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    k_gen_runs_toggle<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(mask, parity_counts, n, threshold, seed);
    note_launch();
    return cudaGetLastError();
}

// Alternating runs, step 2: flip a word when an odd number of toggles precede it.
__global__ void k_gen_runs_apply(uint32_t* mask, const uint64_t* parity_offsets, uint64_t n)
{
    const uint64_t nw = (n + 31) / 32;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t w = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w < nw; w += stride) {
        uint32_t m = mask[w];
        if (parity_offsets[w] & 1ull) m = ~m;
        if (w == nw - 1 && (n & 31u)) m &= (1u << (n & 31u)) - 1u;
        mask[w] = m;
    }
}

cudaError_t launch_gen_runs_apply(uint32_t* mask, const uint64_t* parity_offsets, uint64_t n, int num_sms,
                                  cudaStream_t stream)
{
    const uint64_t nw = (n + 31) / 32;
    uint64_t blocks = (nw + 255) / 256;
    const uint64_t cap = static_cast<uint64_t>(num_sms) * 16;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    k_gen_runs_apply<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(mask, parity_offsets, n);
    note_launch();
    return cudaGetLastError();
}

__global__ void k_gen_mask_dense_prefix(uint32_t* mask, uint64_t n, uint64_t k)
{
    const uint64_t nw = (n + 31) / 32;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t w = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w < nw; w += stride) {
        const uint64_t lo = w * 32;
        uint32_t m;
        if (lo + 32 <= k) m = 0xffffffffu;
        else if (lo >= k) m = 0u;
        else m = (1u << (k - lo)) - 1u;
        mask[w] = m;
    }
}

cudaError_t launch_gen_mask_dense_prefix(uint32_t* mask, uint64_t n, uint64_t k, int num_sms, cudaStream_t stream)
{
    const uint64_t nw = (n + 31) / 32;
    uint64_t blocks = (nw + 255) / 256;
    const uint64_t cap = static_cast<uint64_t>(num_sms) * 16;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    k_gen_mask_dense_prefix<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(mask, n, k);
    note_launch();
    return cudaGetLastError();
}

// Periodic mask: bit i = bit (i % L) of pattern (the selection of compressstore_pattern as
// a mask in memory; the reference builds it MSB-first on the host, generate_mask_pattern,
// src/data_generator.cuh:113-128).
__global__ void k_gen_mask_pattern(uint32_t* mask, uint64_t n, uint32_t pattern, uint32_t L)
{
    const uint64_t nw = (n + 31) / 32;
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t w = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; w < nw; w += stride) {
        uint32_t m = 0;
        uint32_t ph = static_cast<uint32_t>((w * 32) % L);
#pragma unroll 4
        for (uint32_t b = 0; b < 32; ++b) {
            m |= ((pattern >> ph) & 1u) << b;
            if (++ph == L) ph = 0;
        }
        const uint64_t lo = w * 32;
        if (lo + 32 > n) m &= (1u << (n - lo)) - 1u;
        mask[w] = m;
    }
}

cudaError_t launch_gen_mask_pattern(uint32_t* mask, uint64_t n, uint32_t pattern, uint32_t L, int num_sms,
                                    cudaStream_t stream)
{
    const uint64_t nw = (n + 31) / 32;
    uint64_t blocks = (nw + 255) / 256;
    const uint64_t cap = static_cast<uint64_t>(num_sms) * 16;
    if (blocks > cap) blocks = cap;
    if (blocks == 0) blocks = 1;
    k_gen_mask_pattern<<<static_cast<unsigned>(blocks), 256, 0, stream>>>(mask, n, pattern, L);
    note_launch();
    return cudaGetLastError();
}

} // namespace cs
