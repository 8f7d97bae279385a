// cs_internal.cuh — shared definitions of the compaction library: workspace layout,
// look-back status words, kernel parameter blocks and launcher declarations.
#pragma once
#include <cstddef>
#include <cstdint>
#include <utility>
#include <cuda_runtime.h>

#include "cs_ptx.cuh"

namespace cs {

// ---------------------------------------------------------------------------------
// Workspace. One workspace serves one call at a time (stream-ordered reuse only).
//
//   [0, 256)          ws_header
//   [256, ...)        per-call regions: compaction tile statuses, scan tile statuses,
//                     chunk counts (u32), chunk offsets (u64) — laid out by plan_layout.
//
// Look-back statuses are 64-bit words  epoch:22 | flag:2 | value:40.  A status is valid
// only if its epoch equals the header's current epoch, so no per-call clearing pass is
// needed: the last CTA of every look-back kernel advances the epoch. Epochs live in
// [EPOCH_MIN, EPOCH_MAX]; the lower bound keeps any u32/u64 count or offset left in the
// workspace by an earlier call from ever decoding as a valid status (their bits 42..63
// are below 2^7). On wrap the workspace after the header is cleared, except the results
// of the call that wrapped.
// ---------------------------------------------------------------------------------
constexpr uint32_t WS_MAGIC = 0x43535753u; // "CSWS"
constexpr uint32_t EPOCH_MIN = 128u;
constexpr uint32_t EPOCH_MAX = (1u << 22) - 1u;
constexpr uint64_t STATUS_VALUE_MASK = (1ull << 40) - 1ull;
constexpr uint32_t FLAG_AGG = 1u;
constexpr uint32_t FLAG_PREFIX = 2u;
constexpr uint32_t FLAG_POISON = 3u;   // predecessor chain broken by a timed-out wait
constexpr uint64_t POISON = ~0ull;     // offset value meaning "do not write"
constexpr uint64_t COUNT_ERROR = ~0ull; // count written when a bounded wait gave up (CS_COUNT_ERROR)

// Device error codes recorded in ws_header::err (first error wins).
constexpr uint32_t DEVERR_LOOKBACK_TIMEOUT = 1u;
constexpr uint32_t DEVERR_PIPELINE_TIMEOUT = 2u;
constexpr uint32_t DEVERR_RANGE = 3u;

// Pass 1 writes one "saw a sparse block" flag word per CTA into this many slots.
constexpr uint32_t POPC_FLAG_SLOTS = 2048u;

struct alignas(256) ws_header {
    uint32_t magic;
    uint32_t epoch;             // current look-back epoch
    uint32_t err;               // first device error since the last check (sticky)
    uint32_t poison_epoch;      // epoch of the latest call in which a tile poisoned
    uint32_t tile_counter;      // dynamic tile ids, 1-pass compaction kernel
    uint32_t done_counter;      // CTAs finished, 1-pass compaction kernel
    uint32_t scan_tile_counter; // dynamic tile ids, look-back scan kernel
    uint32_t scan_done_counter; // CTAs finished, look-back scan kernel
    uint64_t ws_bytes;          // total workspace bytes (for the wrap clear)
    uint32_t scan_ok_epoch;     // epoch of the latest scan that completed with no poisoned tile
    uint32_t sparse_epoch;      // epoch of the latest pass 1 that saw a sparse 16K block
    uint32_t popc_ctas;         // CTAs of the latest pass 1 (entries of its flag array)
    uint32_t reserved0;
    uint64_t count_word;        // a count slot inside the header: a caller that points d_count here
                                // reads count and error word back with one copy of the header
    uint64_t reserved1[24];
};
static_assert(sizeof(ws_header) == 256, "ws_header must be 256 bytes");

__host__ __device__ __forceinline__ uint64_t pack_status(uint32_t epoch, uint32_t flag, uint64_t value)
{
    return (static_cast<uint64_t>(epoch) << 42) | (static_cast<uint64_t>(flag) << 40) | (value & STATUS_VALUE_MASK);
}
__host__ __device__ __forceinline__ uint32_t status_epoch(uint64_t s)
{
    return static_cast<uint32_t>(s >> 42);
}
__host__ __device__ __forceinline__ uint32_t status_flag(uint64_t s)
{
    return static_cast<uint32_t>(s >> 40) & 3u;
}
__host__ __device__ __forceinline__ uint64_t status_value(uint64_t s)
{
    return s & STATUS_VALUE_MASK;
}

__device__ __forceinline__ void record_error(ws_header* hdr, uint32_t code)
{
    if (hdr) atomicCAS(&hdr->err, 0u, code);
}

// ---------------------------------------------------------------------------------
// Decoupled look-back, executed by ONE full warp for tile `tile` whose own aggregate is
// `agg`. Publishes AGG then PREFIX for this tile and returns the exclusive prefix (the
// sum of the aggregates of all earlier tiles), or POISON if a predecessor's chain is
// broken or the bounded wait ran out (then this tile publishes POISON too, so its
// successors never wait on it and never write with a wrong offset).
// One round covers 32*K predecessors: load k of lane l reads the predecessor at distance
// 32k + l, so each load instruction of the warp touches 256 contiguous bytes (two L2
// lines). K = 1 is the default because wider windows measured slower in the 1-pass kernel
// (n = 2^28 float32 on B200: 4038 GB/s at K = 1, 3592 at K = 4, 3422 at K = 8, 3048 at
// K = 16): every SM's scanner polls the same few status lines, and polling traffic, not
// the number of rounds, sets the look-back latency there.
// With AGG_PUBLISHED the caller has already published the tile's aggregate through
// publish_aggregate (PREFIX for tile 0), and only the look-back and the PREFIX remain.
// ---------------------------------------------------------------------------------
__device__ __forceinline__ void publish_aggregate(uint64_t* status, uint64_t tile, uint64_t agg, uint32_t epoch)
{
    st_relaxed_gpu(&status[tile], pack_status(epoch, tile == 0 ? FLAG_PREFIX : FLAG_AGG, agg));
}

template <int K = 1, bool AGG_PUBLISHED = false>
__device__ __forceinline__ uint64_t lookback_warp(uint64_t* status, uint64_t tile, uint64_t agg, uint32_t epoch,
                                                  uint64_t timeout_ns, ws_header* hdr, uint32_t lane)
{
    if (tile == 0) {
        if (!AGG_PUBLISHED && lane == 0) st_relaxed_gpu(&status[0], pack_status(epoch, FLAG_PREFIX, agg));
        return 0;
    }
    if (!AGG_PUBLISHED && lane == 0) st_relaxed_gpu(&status[tile], pack_status(epoch, FLAG_AGG, agg));

    uint64_t excl = 0;
    int64_t pred = static_cast<int64_t>(tile) - 1; // nearest predecessor of this round
    bool poisoned = false;
    uint64_t t0 = 0;
    uint32_t spins = 0;
    while (true) {
        uint64_t st[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int64_t idx = pred - (32 * k + static_cast<int64_t>(lane));
            st[k] = idx >= 0 ? ld_relaxed_gpu(&status[idx]) : 0ull;
        }
        // nearest PREFIX/POISON in the window (entries past tile 0 act as PREFIX(0)), as
        // (row k, lane); rows before it and lanes before it in its row must all be valid
        uint32_t frow = K, flane = 32, bad = 0, poison = 0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int64_t idx = pred - (32 * k + static_cast<int64_t>(lane));
            const bool real = idx >= 0;
            const uint32_t flag = real ? status_flag(st[k]) : FLAG_PREFIX;
            const bool valid = !real || (status_epoch(st[k]) == epoch && flag != 0u);
            const uint32_t pm = __ballot_sync(0xffffffffu, valid && flag >= FLAG_PREFIX);
            const uint32_t im = __ballot_sync(0xffffffffu, !valid);
            const uint32_t xm = __ballot_sync(0xffffffffu, valid && real && flag == FLAG_POISON);
            if (frow == K) {
                if (pm) {
                    frow = k;
                    flane = __ffs(pm) - 1;
                    const uint32_t upto = flane == 31u ? 0xffffffffu : ((2u << flane) - 1u);
                    bad |= im & upto;
                    poison = xm & (1u << flane);
                } else {
                    bad |= im;
                }
            }
        }
        if (bad == 0u) {
            if (poison) {
                poisoned = true;
                break;
            }
            uint64_t sum = 0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int64_t idx = pred - (32 * k + static_cast<int64_t>(lane));
                const bool use = idx >= 0 && (static_cast<uint32_t>(k) < frow ||
                                              (static_cast<uint32_t>(k) == frow && lane <= flane));
                sum += use ? status_value(st[k]) : 0ull;
            }
            excl += warp_sum64(sum);
            if (frow < K) break;
            pred -= 32 * K;
            continue;
        }
        // some needed predecessor has not published yet: back off, bounded in time (the
        // verdict is made warp-uniform before anyone leaves the loop)
        if (spins == 0) t0 = globaltimer_ns();
        ++spins;
        const bool expired = ((spins & 63u) == 0u) && (globaltimer_ns() - t0 > timeout_ns);
        if (__any_sync(0xffffffffu, expired)) {
            if (lane == 0) record_error(hdr, DEVERR_LOOKBACK_TIMEOUT);
            poisoned = true;
            break;
        }
        __nanosleep(spins < 16 ? 20 : 200);
    }
    poisoned = __shfl_sync(0xffffffffu, poisoned, 0);
    if (poisoned) {
        if (lane == 0) {
            st_relaxed_gpu(&status[tile], pack_status(epoch, FLAG_POISON, 0));
            if (hdr) *reinterpret_cast<volatile uint32_t*>(&hdr->poison_epoch) = epoch;
        }
        return POISON;
    }
    if (lane == 0) st_relaxed_gpu(&status[tile], pack_status(epoch, FLAG_PREFIX, excl + agg));
    return excl;
}

// ---------------------------------------------------------------------------------
// Decoupled look-back executed by a whole CTA of NT threads (NT a multiple of 32): thread
// i inspects predecessor tile-1-i, so one round covers NT predecessors instead of 32. Same
// contract as lookback_warp: publishes AGG then PREFIX (or POISON) for `tile` and returns
// the exclusive prefix or POISON, identically in every thread. Every decision is taken
// from shared memory by all threads alike, so the barriers inside are reached uniformly;
// the caller must not hold other threads at a barrier meanwhile (call it with the whole
// CTA). Used by the scan kernels, whose other warps would otherwise idle at a barrier
// while one warp walks the predecessors 32 at a time.
// ---------------------------------------------------------------------------------
template <int NW>
struct LookbackSmem {
    uint32_t first[NW];   // per warp: lowest thread whose predecessor holds PREFIX/POISON
    uint32_t invalid[NW]; // per warp: lanes whose predecessor has not published
    uint32_t poison[NW];  // per warp: lanes whose predecessor is POISON
    uint64_t sum[NW];     // per warp: partial sums of the used values
};

template <int NT>
__device__ __forceinline__ uint64_t lookback_cta(uint64_t* status, uint64_t tile, uint64_t agg, uint32_t epoch,
                                                 uint64_t timeout_ns, ws_header* hdr, LookbackSmem<NT / 32>& sm)
{
    constexpr int NW = NT / 32;
    constexpr uint32_t NONE = 0xffffffffu;
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    if (tile == 0) {
        if (tid == 0) st_relaxed_gpu(&status[0], pack_status(epoch, FLAG_PREFIX, agg));
        return 0;
    }
    if (tid == 0) st_relaxed_gpu(&status[tile], pack_status(epoch, FLAG_AGG, agg));

    uint64_t excl = 0;
    int64_t pred = static_cast<int64_t>(tile) - 1; // nearest predecessor of this round
    bool poisoned = false;
    uint64_t t0 = 0;
    uint32_t spins = 0;
    while (true) {
        const int64_t idx = pred - static_cast<int64_t>(tid);
        uint64_t s = 0;
        bool valid = true;
        uint32_t flag = FLAG_PREFIX; // threads past tile 0 act as PREFIX(0)
        if (idx >= 0) {
            s = ld_relaxed_gpu(&status[idx]);
            flag = status_flag(s);
            valid = (status_epoch(s) == epoch) && flag != 0u;
        }
        const uint32_t pmask = __ballot_sync(0xffffffffu, valid && flag >= FLAG_PREFIX);
        const uint32_t imask = __ballot_sync(0xffffffffu, !valid);
        const uint32_t xmask = __ballot_sync(0xffffffffu, valid && flag == FLAG_POISON && idx >= 0);
        if (lane == 0) {
            sm.first[warp] = pmask ? warp * 32u + (__ffs(pmask) - 1u) : NONE;
            sm.invalid[warp] = imask;
            sm.poison[warp] = xmask;
        }
        __syncthreads();
        uint32_t first = NONE;
#pragma unroll
        for (int w = 0; w < NW; ++w) first = min(first, sm.first[w]);
        // threads 0..first must all be valid (all threads when no PREFIX is in the window)
        bool missing = false, poison = false;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const uint32_t lo = static_cast<uint32_t>(w) * 32u;
            uint32_t need;
            if (first == NONE || first >= lo + 31u) need = 0xffffffffu;
            else if (first < lo) need = 0u;
            else need = (2u << (first - lo)) - 1u; // lanes 0 .. first-lo
            missing |= (sm.invalid[w] & need) != 0u;
            poison |= (sm.poison[w] & need) != 0u;
        }
        if (!missing) {
            if (poison) {
                poisoned = true;
                break;
            }
            const uint64_t v = ((first == NONE || tid <= first) && idx >= 0) ? status_value(s) : 0ull;
            const uint64_t ws = warp_sum64(v);
            if (lane == 0) sm.sum[warp] = ws;
            __syncthreads();
            uint64_t tot = 0;
#pragma unroll
            for (int w = 0; w < NW; ++w) tot += sm.sum[w];
            excl += tot;
            if (first != NONE) break;
            pred -= NT;
            __syncthreads(); // sums read before the next round rewrites them
            continue;
        }
        // a needed predecessor has not published: back off, bounded in time (thread 0's
        // clock decides for the whole CTA)
        if (spins == 0) t0 = globaltimer_ns();
        ++spins;
        const bool expired = tid == 0 && ((spins & 63u) == 0u) && (globaltimer_ns() - t0 > timeout_ns);
        if (__syncthreads_or(expired)) {
            if (tid == 0) record_error(hdr, DEVERR_LOOKBACK_TIMEOUT);
            poisoned = true;
            break;
        }
        __nanosleep(spins < 16 ? 20 : 200);
    }
    if (poisoned) {
        if (tid == 0) {
            st_relaxed_gpu(&status[tile], pack_status(epoch, FLAG_POISON, 0));
            if (hdr) *reinterpret_cast<volatile uint32_t*>(&hdr->poison_epoch) = epoch;
        }
        return POISON;
    }
    if (tid == 0) st_relaxed_gpu(&status[tile], pack_status(epoch, FLAG_PREFIX, excl + agg));
    return excl;
}

__host__ __device__ __forceinline__ uint32_t prev_epoch(uint32_t e)
{
    return e == EPOCH_MIN ? EPOCH_MAX : e - 1u;
}

// End of a look-back kernel, in two steps. epilogue_ticket (every CTA, all threads) counts
// the CTA as finished and returns, uniformly within the CTA, whether it was the last one.
// epilogue_last (the last CTA only, all its threads) resets the dynamic tile counter,
// records (for a scan) whether the call completed without a poisoned tile, folds pass 1's
// per-CTA sparse flags into the header and advances the epoch. On wrap it clears the
// workspace after the header except [keep_begin, keep_end), the results of this call.
__device__ __forceinline__ bool epilogue_ticket(uint32_t* done_counter, uint32_t* smem_flag)
{
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const uint32_t prev = atomicAdd(done_counter, 1u);
        *smem_flag = (prev == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    const bool last = *smem_flag != 0u;
    if (last) __threadfence();
    return last;
}

__device__ __forceinline__ void epilogue_last(ws_header* hdr, uint32_t* tile_counter, uint32_t* done_counter,
                                              bool is_scan, uint64_t keep_begin, uint64_t keep_end,
                                              const uint32_t* popc_flags)
{
    volatile ws_header* vh = hdr;
    const uint32_t cur = vh->epoch;
    uint32_t next = cur + 1u;
    if (next > EPOCH_MAX) {
        uint4* p = reinterpret_cast<uint4*>(hdr);
        const uint64_t n16 = hdr->ws_bytes / 16u;
        const uint64_t k0 = keep_begin / 16u, k1 = (keep_end + 15u) / 16u;
        for (uint64_t i = sizeof(ws_header) / 16u + threadIdx.x; i < n16; i += blockDim.x)
            if (i < k0 || i >= k1) p[i] = make_uint4(0, 0, 0, 0);
        __threadfence();
        next = EPOCH_MIN;
    }
    // fold pass 1's per-CTA sparse flags (written before this point of the call)
    uint32_t any_sparse = 0;
    if (popc_flags) {
        const uint32_t nctas = vh->popc_ctas;
        const uint32_t nf = nctas < 2048u ? nctas : 2048u; // POPC_FLAG_SLOTS
        for (uint32_t i = threadIdx.x; i < nf; i += blockDim.x) any_sparse |= (popc_flags[i] == cur) ? 1u : 0u;
    }
    any_sparse = __syncthreads_or(any_sparse);
    if (threadIdx.x == 0) {
        if (any_sparse) vh->sparse_epoch = cur;
        if (is_scan && vh->poison_epoch != cur) vh->scan_ok_epoch = cur; // == prev_epoch(next)
        // a new epoch cycle must not meet an old cycle's poison mark (0 is no epoch)
        if (next == EPOCH_MIN) vh->poison_epoch = 0u;
        *tile_counter = 0u;
        *done_counter = 0u;
        vh->epoch = next;
        __threadfence();
    }
}

// epilogue_last for the reduce-then-scan pass (the last CTA, all its threads): `cur` is the
// epoch the kernel read at its start, `any_sparse` whether a CTA saw a sparse block and
// `clean` whether every CTA's waits completed (the pass has no look-back; only the streaming
// form waits, on its own copies). Same wrap clear as epilogue_last.
__device__ __forceinline__ void epilogue_last_blocks(ws_header* hdr, uint32_t cur, bool any_sparse,
                                                     uint64_t keep_begin, uint64_t keep_end, bool clean)
{
    uint32_t next = cur + 1u;
    if (next > EPOCH_MAX) {
        uint4* q = reinterpret_cast<uint4*>(hdr);
        const uint64_t n16 = hdr->ws_bytes / 16u;
        const uint64_t k0 = keep_begin / 16u, k1 = (keep_end + 15u) / 16u;
        for (uint64_t i = sizeof(ws_header) / 16u + threadIdx.x; i < n16; i += blockDim.x)
            if (i < k0 || i >= k1) q[i] = make_uint4(0, 0, 0, 0);
        __threadfence();
        next = EPOCH_MIN;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile ws_header* vh = hdr;
        if (any_sparse) vh->sparse_epoch = cur;
        if (clean) vh->scan_ok_epoch = cur;
        if (next == EPOCH_MIN) vh->poison_epoch = 0u;
        vh->scan_tile_counter = 0u;
        vh->scan_done_counter = 0u;
        vh->epoch = next;
    }
}

// Both steps, for kernels with nothing to do between them.
__device__ __forceinline__ void lookback_kernel_epilogue(ws_header* hdr, uint32_t* tile_counter, uint32_t* done_counter,
                                                         uint32_t* smem_flag, bool is_scan, uint64_t keep_begin,
                                                         uint64_t keep_end, const uint32_t* popc_flags = nullptr)
{
    if (epilogue_ticket(done_counter, smem_flag))
        epilogue_last(hdr, tile_counter, done_counter, is_scan, keep_begin, keep_end, popc_flags);
}

// True when pass 1 of this call saw a block sparse enough for the gather kernel (recorded
// by the scan that followed it, which advanced the epoch).
__device__ __forceinline__ bool last_popc_saw_sparse(const ws_header* hdr)
{
    if (!hdr) return true;
    const volatile ws_header* vh = hdr;
    return vh->sparse_epoch == prev_epoch(vh->epoch);
}

// Header flags a kernel needs, read ONCE per CTA by thread 0 with plain loads (they were
// written by earlier kernels) and shared through shared memory: thousands of threads
// re-reading one line with volatile loads serialise in L2. bit 0: the last scan completed
// cleanly; bit 1: pass 1 of this call saw a sparse block. Call with all threads.
__device__ __forceinline__ uint32_t cta_header_flags(const ws_header* hdr, uint32_t* smem_slot)
{
    if (threadIdx.x == 0) {
        uint32_t f = 3u;
        if (hdr) {
            const uint32_t e = hdr->epoch;
            f = (hdr->scan_ok_epoch == prev_epoch(e) ? 1u : 0u) | (hdr->sparse_epoch == prev_epoch(e) ? 2u : 0u);
        }
        *smem_slot = f;
    }
    __syncthreads();
    return *smem_slot;
}

// True when the look-back scan that ran last on this workspace (stream-ordered before the
// caller) completed with every tile's prefix valid.
__device__ __forceinline__ bool last_scan_ok(const ws_header* hdr)
{
    if (!hdr) return true;
    const volatile ws_header* vh = hdr;
    return vh->scan_ok_epoch == prev_epoch(vh->epoch);
}

// ---------------------------------------------------------------------------------
// Kernel parameters
// ---------------------------------------------------------------------------------

// Pass 1 + 2 of the 3-pass form works in blocks of 2^18 elements (64 chunks of 4096, 128 of
// 2048, 256 of 1024): chunk offsets within a block, plus one prefix per block.
constexpr uint32_t SCAN_BLOCK_LOG2 = 18;

// One column of a batch (or the only column of a plain call), as the device sees it.
struct ColumnDesc {
    const uint8_t* in;
    const uint32_t* mask;
    uint8_t* out;
    uint64_t n;
    uint64_t* d_count;  // the column's selected count (pass 2 writes it)
    uint64_t* offsets;  // the column's chunk offsets (pass 2 writes them)
    const uint64_t* blk_base; // null: offsets are exclusive prefixes of the column; else they
                              // are relative to their 2^18-element block, whose exclusive
                              // prefix is blk_base[chunk >> (SCAN_BLOCK_LOG2 - chunk_log2)]
    uint64_t unit_base; // first TMA unit of the column in its width's unit list (the 1-pass
                        // list for a 1-pass column; also the base of its look-back statuses)
    uint64_t tile_base; // first fused-scan tile of the column (also its status index base)
    uint64_t item_base; // first sparse-kernel item of the column
    uint32_t elem_bytes;
    uint32_t one_pass;  // batch: the column takes the 1-pass form (no pass-1/2 work)
};

// The column a unit/tile/item belongs to: `cols` null means the single column `col0`.
__device__ __forceinline__ const ColumnDesc& column_of(const ColumnDesc& col0, const ColumnDesc* cols,
                                                      const uint32_t* index_col, uint64_t idx)
{
    return cols ? cols[__ldg(index_col + idx)] : col0;
}

// Exclusive output offset of chunk c (chunk length 2^chunk_log2) of a column, from pass 2's
// flat offsets or from the block-relative offsets plus the block's prefix.
__device__ __forceinline__ uint64_t chunk_offset(const ColumnDesc& C, uint64_t c, uint32_t chunk_log2)
{
    const uint64_t o = C.offsets[c];
    return C.blk_base ? o + C.blk_base[c >> (SCAN_BLOCK_LOG2 - chunk_log2)] : o;
}

struct CompactParams {
    ColumnDesc col0;               // the column (cols null); unit_base 0
    uint64_t num_tiles;            // number of look-back units (UNIT_TILES tiles each) of this launch
    ws_header* hdr;
    uint64_t* status;              // 1-pass: one status per unit
    uint64_t sparse_max;           // 3-pass hybrid: units with at most this many selected
                                   // elements belong to the sparse kernel (0: none)
    uint32_t chunk_log2;           // 3-pass: log2(chunk length)
    uint32_t skip;                 // 1: skip payload loads of empty segments
    uint64_t timeout_ns;
    // batch: when cols is set, unit u of this launch belongs to column cols[unit_col[u]] and
    // col0 is unused. 1-pass: a column's units are consecutive in the launch's list, from
    // cols[.].unit_base; their look-back statuses are status[unit_base + unit of the column],
    // and each column's look-back ends at its own first unit.
    const ColumnDesc* cols;
    const uint32_t* unit_col;
    uint64_t keep_begin; // 1-pass: byte range of the workspace the epoch-wrap clear keeps (a
    uint64_t keep_end;   // plan's descriptors and maps); empty for the plain call
};

struct ScanParams {
    const uint32_t* counts;
    uint64_t count;
    uint64_t* offsets;
    uint64_t* total;   // may be null
    ws_header* hdr;
    uint64_t* status;
    uint64_t num_tiles;
    uint64_t timeout_ns;
    uint64_t keep_begin;  // byte range of this call's results inside the workspace,
    uint64_t keep_end;    // preserved by the epoch-wrap clear
    const uint32_t* popc_flags; // pass 1's per-CTA sparse flags (null: none)
};

// Pass 1 + 2 as one reduce-then-scan kernel (chunk length 128 .. 4096, 16-byte aligned
// masks): block b of the flat block list belongs to cols[blk_col[b]] (cols null: col0, whose
// blocks are 0 .. ). Each CTA writes its blocks' block-relative chunk offsets and block sums;
// the last CTA turns the sums into per-column block prefixes and counts.
struct BlockScanParams {
    ColumnDesc col0;
    const ColumnDesc* cols;
    const uint32_t* blk_col;
    uint32_t* item_flags;     // non-null: the 16K-element items of units with at most 1/32
                              // selected (hybrid writeout) get the current epoch here
    uint64_t num_blocks;      // over all columns
    uint64_t* blk_sum;        // [num_blocks] scratch
    uint64_t* blk_base;       // [num_blocks] result: exclusive prefix of each block in its column
    ws_header* hdr;
    uint32_t chunk_log2;
    uint32_t pad;
    uint64_t keep_begin;      // byte range of this call's results inside the workspace,
    uint64_t keep_end;        // preserved by the epoch-wrap clear
};

// Predicate compaction, mask pass (cs_predicate.cu): bs.col0 is the column (its mask is
// `mask`, written by the kernel); lo and hi hold the comparison's bounds as bit patterns of
// the element type in their low bytes (lo_incl, hi_incl and negate describe the same
// selection in bounds form).
struct PredParams {
    BlockScanParams bs;
    const uint8_t* in;
    uint32_t* mask;
    uint64_t lo, hi;
    uint32_t lo_incl, hi_incl, negate, pad;
};

// Last CTA of a reduce-then-scan pass (all 256 threads): turns the block sums into the
// exclusive prefix of every block within its column (blk_base) and writes every column's
// count, or CS_COUNT_ERROR when the pass is not `clean`. s_scan: 8 words of shared memory.
__device__ __forceinline__ void blocks_last_cta(const BlockScanParams& p, uint64_t* s_scan, bool clean)
{
    const uint32_t tid = threadIdx.x;
    const uint32_t lane = tid & 31u;
    const uint32_t warp = tid >> 5;
    // flat exclusive scan of the block sums (ascending, into blk_base); a thread takes V
    // consecutive sums per round so up to 1024 blocks (2^28 elements) need one round
    constexpr uint32_t V = 4;
    const uint64_t T = p.num_blocks;
    uint64_t carry = 0;
    for (uint64_t base = 0; base < T; base += 256 * V) {
        const uint64_t t0 = base + static_cast<uint64_t>(tid) * V;
        uint64_t v[V];
#pragma unroll
        for (uint32_t k = 0; k < V; ++k) v[k] = t0 + k < T ? __ldcg(p.blk_sum + t0 + k) : 0ull;
        uint64_t mine = 0;
#pragma unroll
        for (uint32_t k = 0; k < V; ++k) mine += v[k];
        const uint64_t x = warp_incl_scan64(mine, lane);
        if (lane == 31) s_scan[warp] = x;
        __syncthreads();
        uint64_t run = carry + x - mine, tot = 0;
#pragma unroll
        for (int w = 0; w < 8; ++w) {
            const uint64_t y = s_scan[w];
            run += (static_cast<uint32_t>(w) < warp) ? y : 0ull;
            tot += y;
        }
#pragma unroll
        for (uint32_t k = 0; k < V; ++k) {
            if (t0 + k < T) p.blk_base[t0 + k] = run;
            run += v[k];
        }
        carry += tot;
        __syncthreads();
    }
    if (!p.cols) {
        // one column: its first block is block 0, so the flat prefixes are final
        if (tid == 0) *p.col0.d_count = clean ? carry : COUNT_ERROR;
    } else {
        // descending rounds: the prefix of each block relative to its column's first block
        // (all reads of a round precede its writes, and a column's first block is never in a
        // later round), and each column's count at its last block
        const uint64_t last_base = ((T - 1) / (256 * V)) * (256 * V);
        for (int64_t base = static_cast<int64_t>(last_base); base >= 0; base -= 256 * V) {
            const uint64_t t0 = static_cast<uint64_t>(base) + static_cast<uint64_t>(tid) * V;
            uint64_t res[V]; // prefix of the block within its column
#pragma unroll
            for (uint32_t k = 0; k < V; ++k) {
                const uint64_t t = t0 + k;
                res[k] = 0;
                if (t < T) {
                    const ColumnDesc& c = p.cols[__ldg(p.blk_col + t)];
                    res[k] = __ldcg(p.blk_base + t) - __ldcg(p.blk_base + c.tile_base);
                    const uint64_t col_blocks = (c.n + (1ull << SCAN_BLOCK_LOG2) - 1) >> SCAN_BLOCK_LOG2;
                    // counts never alias blk_base: written before the round's barrier
                    if (t - c.tile_base == col_blocks - 1)
                        *c.d_count = clean ? res[k] + __ldcg(p.blk_sum + t) : COUNT_ERROR;
                }
            }
            __syncthreads();
#pragma unroll
            for (uint32_t k = 0; k < V; ++k)
                if (t0 + k < T) p.blk_base[t0 + k] = res[k];
            __syncthreads();
        }
    }
}

struct SparseParams {
    ColumnDesc col0;          // single column (cols null)
    const ColumnDesc* cols;   // batch: item t belongs to cols[item_col[t]]
    const uint32_t* item_col;
    uint64_t num_items;       // 16-block items over all columns
    const ws_header* hdr;
    uint32_t chunk_log2;
    const uint32_t* item_flags; // items pass 1 marked with its epoch (the sparse ones); null:
                                // test every item
};

// ---------------------------------------------------------------------------------
// Launchers (defined in the .cu files). All return cudaError_t of the launch.
// ---------------------------------------------------------------------------------
constexpr uint32_t TILE_BYTES = 32768;       // payload bytes per tile of the TMA kernels
#ifndef CS_UNIT_TILES
#define CS_UNIT_TILES 4
#endif
constexpr uint32_t UNIT_TILES = CS_UNIT_TILES; // tiles per look-back unit (one offset per unit)
constexpr uint32_t SCAN_ITEMS_PER_THREAD = 16;
constexpr uint32_t SCAN_THREADS = 256;
constexpr uint32_t SCAN_TILE = SCAN_ITEMS_PER_THREAD * SCAN_THREADS; // 4096 counts

__host__ __device__ constexpr uint32_t tile_elems_for(uint32_t elem_bytes)
{
    return TILE_BYTES / elem_bytes;
}
__host__ __device__ constexpr uint32_t unit_elems_for(uint32_t elem_bytes)
{
    return UNIT_TILES * (TILE_BYTES / elem_bytes);
}

cudaError_t launch_popc_chunks(const uint32_t* mask, uint64_t n, uint32_t chunk_log2, uint32_t* counts,
                               ws_header* hdr, uint32_t* cta_flags, int num_sms, cudaStream_t stream);
cudaError_t launch_scan(const ScanParams& p, int num_sms, cudaStream_t stream);
// Fused pass 1 + pass 2 for chunk length 4096 and a 16-byte-aligned mask.
constexpr uint32_t FUSED_TILE_CHUNKS = 64; // 4096-element chunks per reduce-then-scan block
static_assert(FUSED_TILE_CHUNKS * 4096u == (1u << SCAN_BLOCK_LOG2), "a plan tile is one scan block");
cudaError_t launch_popc_blocks(const BlockScanParams& p, int num_sms, cudaStream_t stream);
cudaError_t launch_pred_mask(const PredParams& p, int type, int op, int num_sms, cudaStream_t stream);
cudaError_t launch_writeout_sparse(const SparseParams& p, int num_sms, cudaStream_t stream);
__host__ __device__ constexpr uint64_t sparse_items_for(uint64_t n)
{
    return ((n + 1023) / 1024 + 15) / 16; // items of 16 blocks of 1024 elements
}
cudaError_t launch_writeout_naive(const void* in, const uint32_t* mask, void* out, uint64_t n, uint32_t elem_bytes,
                                  const uint64_t* chunk_offsets, const uint32_t* chunk_counts, uint32_t chunk_log2,
                                  const ws_header* hdr, int num_sms, cudaStream_t stream);
// mode 0: 1-pass look-back; mode 1: 3-pass (prefix from chunk_offsets); mode 2: 1-pass with a
// deeper payload ring (long columns of 4- and 8-byte elements; mode 0 for narrower ones).
// unit_tiles: tiles per look-back unit, UNIT_TILES or (mode 0 only) 1 for short columns.
cudaError_t launch_compact_tma(const CompactParams& p, uint32_t elem_bytes, int mode, uint32_t grid,
                               cudaStream_t stream, uint32_t unit_tiles = UNIT_TILES);
// Occupancy-derived resident CTAs per SM of the TMA kernel (after its smem attribute is set).
int compact_tma_blocks_per_sm(uint32_t elem_bytes, int mode, uint32_t unit_tiles = UNIT_TILES);
// Dynamic shared memory of one TMA-kernel CTA (its Layout TOTAL); 0 for bad arguments.
uint32_t compact_tma_smem_bytes(uint32_t elem_bytes, int mode, uint32_t unit_tiles = UNIT_TILES);

cudaError_t launch_gen_payload(void* out, uint64_t n, uint32_t elem_bytes, uint64_t seed, int float_unit, int num_sms,
                               cudaStream_t stream);
cudaError_t launch_gen_mask_bernoulli(uint32_t* mask, uint64_t n, uint64_t threshold, uint64_t seed, int num_sms,
                                      cudaStream_t stream);
cudaError_t launch_gen_runs_toggle(uint32_t* mask, uint32_t* parity_counts, uint64_t n, uint64_t threshold,
                                   uint64_t seed, int num_sms, cudaStream_t stream);
cudaError_t launch_gen_runs_apply(uint32_t* mask, const uint64_t* parity_offsets, uint64_t n, int num_sms,
                                  cudaStream_t stream);
cudaError_t launch_gen_mask_dense_prefix(uint32_t* mask, uint64_t n, uint64_t k, int num_sms, cudaStream_t stream);
cudaError_t launch_gen_mask_pattern(uint32_t* mask, uint64_t n, uint32_t pattern, uint32_t L, int num_sms,
                                    cudaStream_t stream);
cudaError_t launch_ws_init(ws_header* hdr, size_t ws_bytes, cudaStream_t stream);

void note_launch(uint64_t k = 1);

// Launch with programmatic stream serialization (programmatic dependent launch): the kernel
// may be scheduled while the previous kernel on the stream drains, and must call
// grid_dependency_wait() before it reads anything earlier kernels produced.
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                       Args&&... args)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

} // namespace cs
