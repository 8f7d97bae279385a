// cs_api.cu — the C ABI (include/compressstore.h): argument checking, workspace layout,
// algorithm resolution, the per-(device, stream) scratch cache of the plain call, and the
// generator / pass entry points.
#include <atomic>
#include <cstdint>
#include <limits>
#include <cstring>
#include <map>
#include <mutex>
#include <utility>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"
#include "cs_tuning.h"

namespace cs {

static std::atomic<uint64_t> g_launches{0};
void note_launch(uint64_t k)
{
    g_launches.fetch_add(k, std::memory_order_relaxed);
}

namespace {

constexpr uint64_t MAX_N = (1ull << 40) - 1; // status words carry 40-bit offsets
// The 1-pass kernel takes one-tile units for a column with fewer full units than SMs and at
// most this many one-tile units (the workspace reserves statuses for that many).
constexpr uint64_t SHORT_UNITS_MAX = 1024;
// ... and the deeper payload ring (mode 2) for 4- and 8-byte columns of at least this many
// full units per SM.
constexpr uint64_t DEEP_UNITS_PER_SM = 16;
constexpr uint64_t DEFAULT_TIMEOUT_NS = 2000000000ull;

struct DeviceInfo {
    int sms = 0;
    int major = 0;
};

std::mutex g_dev_mu;
std::map<int, DeviceInfo> g_dev;

int current_device_info(DeviceInfo* out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CS_ERR_NO_DEVICE;
    {
        std::lock_guard<std::mutex> lk(g_dev_mu);
        auto it = g_dev.find(dev);
        if (it != g_dev.end()) {
            *out = it->second;
            return CS_SUCCESS;
        }
    }
    DeviceInfo di;
    if (cudaDeviceGetAttribute(&di.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return CS_ERR_NO_DEVICE;
    if (cudaDeviceGetAttribute(&di.major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) return CS_ERR_NO_DEVICE;
    if (di.major != 10) return CS_ERR_NO_DEVICE; // built for sm_100a only
    std::lock_guard<std::mutex> lk(g_dev_mu);
    g_dev[dev] = di;
    *out = di;
    return CS_SUCCESS;
}

inline size_t align256(size_t x)
{
    return (x + 255) & ~static_cast<size_t>(255);
}

inline bool is_pow2(uint64_t x)
{
    return x && !(x & (x - 1));
}

inline uint32_t ilog2(uint64_t x)
{
    uint32_t r = 0;
    while ((1ull << r) < x) ++r;
    return r;
}

inline bool aligned(const void* p, uintptr_t a)
{
    return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0;
}

struct Layout {
    uint64_t num_tiles = 0;   // units (UNIT_TILES tiles) of the TMA kernel
    uint64_t num_units1 = 0;  // one-tile units of the 1-pass kernel for short columns
    uint64_t num_chunks = 0;  // popcount chunks
    uint64_t scan_tiles = 0;  // look-back scan tiles over the chunks
    size_t off_status = 0;
    size_t off_scan_status = 0;
    size_t off_counts = 0;
    size_t off_offsets = 0;
    size_t off_blk_base = 0;  // per-2^18-element block prefixes of the reduce-then-scan pass
    size_t off_mask = 0;      // predicate compaction: the selection mask it writes (0: none)
    size_t off_item_flags = 0; // sparse items of the hybrid writeout, marked by pass 1
    size_t off_flags = 0;     // pass 1's per-CTA sparse flags
    size_t total = 0;
};

// All regions every algorithm may need, so AUTO may switch algorithm freely.
Layout plan_layout(uint64_t n, uint32_t elem_bytes, uint32_t chunk_log2, bool with_mask = false)
{
    Layout l;
    const uint64_t ue = unit_elems_for(elem_bytes);
    const uint64_t te = tile_elems_for(elem_bytes);
    l.num_tiles = (n + ue - 1) / ue;
    l.num_units1 = (n + te - 1) / te;
    l.num_chunks = (n + (1ull << chunk_log2) - 1) >> chunk_log2;
    // enough statuses for the plain scan (4096 counts per tile); the reduce-then-scan pass
    // keeps its block sums here too (one per 2^18 elements <= one per 64 chunks)
    l.scan_tiles = (l.num_chunks + FUSED_TILE_CHUNKS - 1) / FUSED_TILE_CHUNKS;
    size_t off = sizeof(ws_header);
    l.off_status = off; // one look-back status per unit, for either unit size a column may take
    const uint64_t short_units = l.num_units1 < SHORT_UNITS_MAX ? l.num_units1 : SHORT_UNITS_MAX;
    off += align256(8 * (l.num_tiles > short_units ? l.num_tiles : short_units));
    l.off_scan_status = off;
    off += align256(8 * l.scan_tiles);
    l.off_counts = off;
    off += align256(4 * l.num_chunks);
    l.off_offsets = off;
    off += align256(8 * l.num_chunks);
    l.off_blk_base = off;
    off += align256(8 * ((n + (1ull << SCAN_BLOCK_LOG2) - 1) >> SCAN_BLOCK_LOG2));
    // inside the range the epoch-wrap clear keeps: later kernels of the call read these
    l.off_item_flags = off;
    off += align256(4 * sparse_items_for(n));
    if (with_mask) {
        l.off_mask = off;
        off += align256(4 * ((n + 31) / 32));
    }
    l.off_flags = off;
    off += align256(4 * POPC_FLAG_SLOTS);
    l.total = align256(off);
    return l;
}

struct Resolved {
    int algo;
    uint32_t chunk_log2;
    uint32_t grid;
    uint32_t skip;
    uint64_t timeout_ns;
};

int resolve_config(const cs_config* cfg, uint64_t n, uint32_t elem_bytes, Resolved* r)
{
    cs_config c{};
    if (cfg) c = *cfg;
    uint32_t L = c.chunk_length ? c.chunk_length : 1024u;
    if (!is_pow2(L) || L < 32 || L > 65536) return CS_ERR_INVALID_VALUE;
    if (c.algo < CS_ALGO_AUTO || c.algo > CS_ALGO_NAIVE) return CS_ERR_INVALID_VALUE;
    if (!(c.selectivity >= 0.0f && c.selectivity <= 1.0f)) return CS_ERR_INVALID_VALUE; // NaN too
    r->algo = c.algo;
    r->chunk_log2 = ilog2(L);
    r->grid = c.grid_dim;
    r->skip = (c.skip == 2) ? 0u : 1u;
    r->timeout_ns = c.timeout_ns ? c.timeout_ns : DEFAULT_TIMEOUT_NS;
    if (r->algo == CS_ALGO_AUTO) {
        const TuneChoice t = tune_lookup(n, elem_bytes, c.selectivity);
        r->algo = t.algo;
        if (!(cfg && cfg->chunk_length)) r->chunk_log2 = ilog2(t.chunk_length);
    }
    return CS_SUCCESS;
}

int check_common(const void* d_in, const void* d_mask, void* d_out, uint64_t n, uint32_t elem_bytes,
                 uint64_t* d_count)
{
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8) return CS_ERR_INVALID_VALUE;
    if (!d_count) return CS_ERR_INVALID_VALUE;
    if (n > MAX_N) return CS_ERR_NOT_SUPPORTED;
    if (n == 0) return CS_SUCCESS;
    if (!d_in || !d_mask || !d_out) return CS_ERR_INVALID_VALUE;
    if (!aligned(d_in, elem_bytes) || !aligned(d_out, elem_bytes) || !aligned(d_mask, 4) || !aligned(d_count, 8))
        return CS_ERR_MISALIGNED;
    return CS_SUCCESS;
}

inline int cuda_status(cudaError_t e)
{
    if (e == cudaSuccess) return CS_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return CS_ERR_OUT_OF_MEMORY;
    return CS_ERR_CUDA;
}

uint32_t persistent_grid(uint32_t elem_bytes, int mode, const DeviceInfo& di, uint64_t num_tiles, uint32_t requested,
                         uint32_t unit_tiles = UNIT_TILES)
{
    uint64_t g = requested;
    if (g == 0) {
        int bps = compact_tma_blocks_per_sm(elem_bytes, mode, unit_tiles);
        if (bps < 1) bps = 1;
        g = static_cast<uint64_t>(bps) * di.sms;
    }
    if (g > num_tiles) g = num_tiles;
    if (g == 0) g = 1;
    return static_cast<uint32_t>(g);
}

ColumnDesc make_column(const void* d_in, const void* d_mask, void* d_out, uint64_t n, uint32_t elem_bytes,
                       uint64_t* d_count, uint64_t* offsets)
{
    ColumnDesc c{};
    c.in = static_cast<const uint8_t*>(d_in);
    c.mask = static_cast<const uint32_t*>(d_mask);
    c.out = static_cast<uint8_t*>(d_out);
    c.n = n;
    c.d_count = d_count;
    c.offsets = offsets;
    c.elem_bytes = elem_bytes;
    return c;
}

// Pass 3 of the 3-pass form over chunk offsets already in the workspace: the sparse gather
// (hybrid only: units with at most 1/32 selected) and the TMA-staged writeout of the rest.
int launch_writeout_3pass(const ColumnDesc& col, const Layout& l, ws_header* hdr, const Resolved& r, bool hybrid,
                          const uint32_t* item_flags, const DeviceInfo& di, cudaStream_t stream)
{
    const uint32_t elem_bytes = col.elem_bytes;
    const uint64_t ue = unit_elems_for(elem_bytes);
    const uint64_t sparse_max = hybrid ? ue / 32 : 0;
    if (hybrid) {
        SparseParams spp{};
        spp.col0 = col;
        spp.num_items = sparse_items_for(col.n);
        spp.hdr = hdr;
        spp.chunk_log2 = r.chunk_log2;
        spp.item_flags = item_flags;
        const cudaError_t e = launch_writeout_sparse(spp, di.sms, stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    CompactParams p{};
    p.col0 = col;
    p.num_tiles = l.num_tiles;
    p.hdr = hdr;
    p.sparse_max = sparse_max;
    p.chunk_log2 = r.chunk_log2;
    p.skip = r.skip;
    p.timeout_ns = r.timeout_ns;
    const uint32_t grid = persistent_grid(elem_bytes, 1, di, l.num_tiles, r.grid);
    return cuda_status(launch_compact_tma(p, elem_bytes, 1, grid, stream));
}

int run_compaction(const void* d_in, const void* d_mask, void* d_out, uint64_t n, uint32_t elem_bytes,
                   uint64_t* d_count, void* d_ws, size_t ws_bytes, const Resolved& r, bool auto_route,
                   cudaStream_t stream)
{
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    const Layout l = plan_layout(n, elem_bytes, r.chunk_log2);
    if (!d_ws || ws_bytes < l.total || !aligned(d_ws, 256)) return CS_ERR_WORKSPACE;
    uint8_t* ws = static_cast<uint8_t*>(d_ws);
    ws_header* hdr = reinterpret_cast<ws_header*>(ws);

    int algo = r.algo;
    const bool tma_ok = aligned(d_in, 16) && aligned(d_out, 16) && aligned(d_mask, 16);
    if ((algo == CS_ALGO_1PASS || algo == CS_ALGO_3PASS) && !tma_ok) {
        if (!auto_route) return CS_ERR_MISALIGNED;
        algo = CS_ALGO_NAIVE;
    }

    if (algo == CS_ALGO_1PASS) {
        // a column with fewer full-size units than SMs takes one-tile units, so that about
        // four times as many SMs share it
        const uint32_t unit_tiles =
            l.num_tiles < static_cast<uint64_t>(di.sms) && l.num_units1 <= SHORT_UNITS_MAX ? 1u : UNIT_TILES;
        CompactParams p{};
        p.col0 = make_column(d_in, d_mask, d_out, n, elem_bytes, d_count, nullptr);
        p.num_tiles = unit_tiles == 1u ? l.num_units1 : l.num_tiles;
        p.hdr = hdr;
        p.status = reinterpret_cast<uint64_t*>(ws + l.off_status);
        p.skip = r.skip;
        p.timeout_ns = r.timeout_ns;
        const int mode = (unit_tiles == UNIT_TILES && elem_bytes >= 4 &&
                          l.num_tiles >= DEEP_UNITS_PER_SM * static_cast<uint64_t>(di.sms))
                             ? 2
                             : 0;
        const uint32_t grid = persistent_grid(elem_bytes, mode, di, p.num_tiles, r.grid, unit_tiles);
        return cuda_status(launch_compact_tma(p, elem_bytes, mode, grid, stream, unit_tiles));
    }

    // 3-pass family: popcount -> prefix sum -> writeout
    uint32_t* counts = reinterpret_cast<uint32_t*>(ws + l.off_counts);
    uint64_t* offsets = reinterpret_cast<uint64_t*>(ws + l.off_offsets);
    uint32_t* flags = reinterpret_cast<uint32_t*>(ws + l.off_flags);
    const uint64_t ue = unit_elems_for(elem_bytes);
    const bool tma_writeout = algo == CS_ALGO_3PASS && (1ull << r.chunk_log2) <= ue;
    // passes 1 + 2 in one reduce-then-scan launch (block-relative offsets + block prefixes)
    const bool blocks = tma_writeout && r.chunk_log2 >= 7 && r.chunk_log2 <= 12 && aligned(d_mask, 16);
    const bool hybrid = algo == CS_ALGO_3PASS && r.chunk_log2 <= 12 && r.skip;
    uint64_t* blk_base = blocks ? reinterpret_cast<uint64_t*>(ws + l.off_blk_base) : nullptr;
    // with the block pass, pass 1 marks the sparse units' items and the gather visits only those
    uint32_t* item_flags = blocks && hybrid ? reinterpret_cast<uint32_t*>(ws + l.off_item_flags) : nullptr;
    cudaError_t e;
    if (blocks) {
        BlockScanParams bp{};
        bp.col0 = make_column(d_in, d_mask, d_out, n, elem_bytes, d_count, offsets);
        bp.col0.blk_base = blk_base;
        bp.num_blocks = (n + (1ull << SCAN_BLOCK_LOG2) - 1) >> SCAN_BLOCK_LOG2;
        bp.blk_sum = reinterpret_cast<uint64_t*>(ws + l.off_scan_status);
        bp.blk_base = blk_base;
        bp.hdr = hdr;
        bp.item_flags = item_flags;
        bp.chunk_log2 = r.chunk_log2;
        bp.keep_begin = l.off_counts;
        bp.keep_end = l.off_flags + 4 * POPC_FLAG_SLOTS;
        e = launch_popc_blocks(bp, di.sms, stream);
        if (e != cudaSuccess) return cuda_status(e);
    } else {
        ScanParams sp{};
        sp.counts = counts;
        sp.count = l.num_chunks;
        sp.offsets = offsets;
        sp.total = d_count;
        sp.hdr = hdr;
        sp.status = reinterpret_cast<uint64_t*>(ws + l.off_scan_status);
        sp.timeout_ns = r.timeout_ns;
        sp.keep_begin = l.off_counts;
        sp.keep_end = l.off_flags + 4 * POPC_FLAG_SLOTS;
        sp.popc_flags = flags;
        e = launch_popc_chunks(static_cast<const uint32_t*>(d_mask), n, r.chunk_log2, counts, hdr, flags, di.sms, stream);
        if (e != cudaSuccess) return cuda_status(e);
        sp.num_tiles = (l.num_chunks + SCAN_TILE - 1) / SCAN_TILE;
        e = launch_scan(sp, di.sms, stream);
        if (e != cudaSuccess) return cuda_status(e);
    }
    ColumnDesc col = make_column(d_in, d_mask, d_out, n, elem_bytes, d_count, offsets);
    col.blk_base = blk_base;
    if (tma_writeout) return launch_writeout_3pass(col, l, hdr, r, hybrid, item_flags, di, stream);
    // chunks longer than a TMA tile, misaligned pointers, or CS_ALGO_NAIVE
    return cuda_status(launch_writeout_naive(d_in, static_cast<const uint32_t*>(d_mask), d_out, n, elem_bytes, offsets,
                                             counts, r.chunk_log2, hdr, di.sms, stream));
}

// ---------------------------------------------------------------------------------
// Library-owned scratch for compressstore / compressstore_cfg / compressstore_if: one
// workspace per (device, stream), grown with stream-ordered allocation so a workspace still
// in use by earlier work on the stream is released only after that work. An entry lives
// until compressstore_release(stream) frees it (a caller that destroys streams calls it
// first; the library cannot tell a destroyed stream's handle from a live one).
// ---------------------------------------------------------------------------------
struct CachedWs {
    void* ptr = nullptr;
    size_t bytes = 0;
};
std::mutex g_ws_mu;
std::map<std::pair<int, cudaStream_t>, CachedWs> g_ws;

int cached_workspace(size_t need, cudaStream_t stream, void** out, size_t* out_bytes)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CS_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_ws_mu);
    CachedWs& c = g_ws[{dev, stream}];
    if (c.bytes < need) {
        size_t want = need < (1u << 20) ? (1u << 20) : need + need / 4;
        want = align256(want);
        void* p = nullptr;
        cudaError_t e = cudaMallocAsync(&p, want, stream);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return CS_ERR_OUT_OF_MEMORY;
        }
        e = launch_ws_init(static_cast<ws_header*>(p), want, stream);
        if (e != cudaSuccess) {
            cudaFreeAsync(p, stream);
            return cuda_status(e);
        }
        if (c.ptr) cudaFreeAsync(c.ptr, stream);
        c.ptr = p;
        c.bytes = want;
    }
    *out = c.ptr;
    *out_bytes = c.bytes;
    return CS_SUCCESS;
}

// Free the cached workspace of (current device, stream), in the stream's order.
int release_cached_workspace(cudaStream_t stream)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CS_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_ws_mu);
    auto it = g_ws.find({dev, stream});
    if (it == g_ws.end()) return CS_SUCCESS;
    const cudaError_t e = it->second.ptr ? cudaFreeAsync(it->second.ptr, stream) : cudaSuccess;
    g_ws.erase(it);
    return cuda_status(e);
}

int lookup_cached_workspace(cudaStream_t stream, void** out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CS_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_ws_mu);
    auto it = g_ws.find({dev, stream});
    if (it == g_ws.end()) {
        *out = nullptr;
        return CS_SUCCESS;
    }
    *out = it->second.ptr;
    return CS_SUCCESS;
}

int check_workspace_error(void* d_ws, cudaStream_t stream)
{
    cudaError_t e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return cuda_status(e);
    if (!d_ws) return CS_SUCCESS;
    uint32_t err = 0;
    ws_header* hdr = static_cast<ws_header*>(d_ws);
    e = cudaMemcpy(&err, &hdr->err, sizeof(err), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(e);
    if (err == 0) return CS_SUCCESS;
    e = cudaMemset(&hdr->err, 0, sizeof(uint32_t));
    if (e != cudaSuccess) return cuda_status(e);
    return err == DEVERR_RANGE ? CS_ERR_INVALID_VALUE : CS_ERR_TIMEOUT;
}

// The predicate as lo (<|<=) x (<|<=) hi, negated for NE; bounds as bit patterns of T.
template <typename T>
void predicate_bounds_t(const cs_predicate& pr, PredParams& pp)
{
    T a, b;
    std::memcpy(&a, &pr.a, sizeof(T));
    std::memcpy(&b, &pr.b, sizeof(T));
    const T lowest = std::numeric_limits<T>::has_infinity ? -std::numeric_limits<T>::infinity()
                                                          : std::numeric_limits<T>::lowest();
    const T highest = std::numeric_limits<T>::has_infinity ? std::numeric_limits<T>::infinity()
                                                           : std::numeric_limits<T>::max();
    T lo = lowest, hi = highest;
    bool li = true, hi_i = true, neg = false;
    switch (pr.op) {
        case CS_PRED_LT: hi = a; hi_i = false; break;
        case CS_PRED_LE: hi = a; break;
        case CS_PRED_GT: lo = a; li = false; break;
        case CS_PRED_GE: lo = a; break;
        case CS_PRED_EQ: lo = hi = a; break;
        case CS_PRED_NE: lo = hi = a; neg = true; break;
        default: lo = a; hi = b; break; // CS_PRED_BETWEEN
    }
    pp.lo = pp.hi = 0;
    std::memcpy(&pp.lo, &lo, sizeof(T));
    std::memcpy(&pp.hi, &hi, sizeof(T));
    pp.lo_incl = li;
    pp.hi_incl = hi_i;
    pp.negate = neg;
}

// Element width of a cs_elem_type and its bounds; 0 for an unknown type.
uint32_t predicate_bounds(const cs_predicate& pr, PredParams& pp)
{
    switch (pr.type) {
        case CS_U8: predicate_bounds_t<uint8_t>(pr, pp); return 1;
        case CS_U16: predicate_bounds_t<uint16_t>(pr, pp); return 2;
        case CS_U32: predicate_bounds_t<uint32_t>(pr, pp); return 4;
        case CS_U64: predicate_bounds_t<uint64_t>(pr, pp); return 8;
        case CS_I8: predicate_bounds_t<int8_t>(pr, pp); return 1;
        case CS_I16: predicate_bounds_t<int16_t>(pr, pp); return 2;
        case CS_I32: predicate_bounds_t<int32_t>(pr, pp); return 4;
        case CS_I64: predicate_bounds_t<int64_t>(pr, pp); return 8;
        case CS_F32: predicate_bounds_t<float>(pr, pp); return 4;
        case CS_F64: predicate_bounds_t<double>(pr, pp); return 8;
        default: return 0;
    }
}

} // namespace
} // namespace cs

using namespace cs;

extern "C" {

size_t compressstore_workspace_size(uint64_t n, uint32_t elem_bytes, const cs_config* cfg)
{
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8) return 0;
    Resolved r{};
    if (resolve_config(cfg, n, elem_bytes, &r) != CS_SUCCESS) return 0;
    return plan_layout(n, elem_bytes, r.chunk_log2).total;
}

int cs_workspace_init(void* d_ws, size_t ws_bytes, cs_stream_t stream)
{
    if (!d_ws || ws_bytes < sizeof(ws_header) || !aligned(d_ws, 256)) return CS_ERR_WORKSPACE;
    return cuda_status(launch_ws_init(static_cast<ws_header*>(d_ws), ws_bytes & ~static_cast<size_t>(15),
                                      reinterpret_cast<cudaStream_t>(stream)));
}

int compressstore_ex(const void* d_in, const void* d_mask, void* d_out, uint64_t n, uint32_t elem_bytes,
                     uint64_t* d_count, void* d_ws, size_t ws_bytes, const cs_config* cfg, cs_stream_t stream)
{
    int st = check_common(d_in, d_mask, d_out, n, elem_bytes, d_count);
    if (st) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (n == 0) return cuda_status(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), s));
    Resolved r{};
    st = resolve_config(cfg, n, elem_bytes, &r);
    if (st) return st;
    const bool auto_route = !(cfg && cfg->algo != CS_ALGO_AUTO);
    return run_compaction(d_in, d_mask, d_out, n, elem_bytes, d_count, d_ws, ws_bytes, r, auto_route, s);
}

int compressstore_cfg(const void* d_in, const void* d_mask, void* d_out, uint64_t n, uint32_t elem_bytes,
                      uint64_t* d_count, const cs_config* cfg, cs_stream_t stream)
{
    int st = check_common(d_in, d_mask, d_out, n, elem_bytes, d_count);
    if (st) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (n == 0) return cuda_status(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), s));
    DeviceInfo di;
    st = current_device_info(&di);
    if (st) return st;
    Resolved r{};
    st = resolve_config(cfg, n, elem_bytes, &r);
    if (st) return st;
    const size_t need = plan_layout(n, elem_bytes, r.chunk_log2).total;
    void* ws = nullptr;
    size_t ws_bytes = 0;
    st = cached_workspace(need, s, &ws, &ws_bytes);
    if (st) return st;
    const bool auto_route = !(cfg && cfg->algo != CS_ALGO_AUTO);
    return run_compaction(d_in, d_mask, d_out, n, elem_bytes, d_count, ws, ws_bytes, r, auto_route, s);
}

int compressstore(const void* d_in, const void* d_mask, void* d_out, uint64_t n, uint32_t elem_bytes,
                  uint64_t* d_count, cs_stream_t stream)
{
    return compressstore_cfg(d_in, d_mask, d_out, n, elem_bytes, d_count, nullptr, stream);
}

int compressstore_if(const void* d_in, void* d_out, uint64_t n, const cs_predicate* pred, uint32_t* d_mask_out,
                     uint64_t* d_count, cs_stream_t stream)
{
    if (!pred || !d_count) return CS_ERR_INVALID_VALUE;
    if (pred->op < CS_PRED_LT || pred->op > CS_PRED_BETWEEN) return CS_ERR_INVALID_VALUE;
    PredParams pp{};
    const uint32_t w = predicate_bounds(*pred, pp);
    if (w == 0) return CS_ERR_INVALID_VALUE;
    if (n > MAX_N) return CS_ERR_NOT_SUPPORTED;
    if (!aligned(d_count, 8)) return CS_ERR_MISALIGNED;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (n == 0) return cuda_status(cudaMemsetAsync(d_count, 0, sizeof(uint64_t), s));
    if (!d_in || !d_out) return CS_ERR_INVALID_VALUE;
    if (!aligned(d_in, 16) || !aligned(d_out, 16) || (d_mask_out && !aligned(d_mask_out, 16))) return CS_ERR_MISALIGNED;
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    Resolved r{};
    r.algo = CS_ALGO_3PASS;
    r.chunk_log2 = 12; // one chunk per 4096-element row of the predicate pass
    r.grid = 0;
    r.skip = 1;
    r.timeout_ns = DEFAULT_TIMEOUT_NS;
    const Layout l = plan_layout(n, w, r.chunk_log2, d_mask_out == nullptr);
    void* ws = nullptr;
    size_t ws_bytes = 0;
    st = cached_workspace(l.total, s, &ws, &ws_bytes);
    if (st) return st;
    uint8_t* wsb = static_cast<uint8_t*>(ws);
    ws_header* hdr = reinterpret_cast<ws_header*>(wsb);
    uint32_t* mask = d_mask_out ? d_mask_out : reinterpret_cast<uint32_t*>(wsb + l.off_mask);
    uint64_t* offsets = reinterpret_cast<uint64_t*>(wsb + l.off_offsets);
    uint64_t* blk_base = reinterpret_cast<uint64_t*>(wsb + l.off_blk_base);
    ColumnDesc col = make_column(d_in, mask, d_out, n, w, d_count, offsets);
    col.blk_base = blk_base;
    pp.bs.col0 = col;
    pp.bs.num_blocks = (n + (1ull << SCAN_BLOCK_LOG2) - 1) >> SCAN_BLOCK_LOG2;
    pp.bs.blk_sum = reinterpret_cast<uint64_t*>(wsb + l.off_scan_status);
    pp.bs.blk_base = blk_base;
    pp.bs.hdr = hdr;
    pp.bs.item_flags = reinterpret_cast<uint32_t*>(wsb + l.off_item_flags);
    pp.bs.chunk_log2 = r.chunk_log2;
    pp.bs.keep_begin = l.off_counts;
    pp.bs.keep_end = l.off_flags + 4 * POPC_FLAG_SLOTS;
    pp.in = static_cast<const uint8_t*>(d_in);
    pp.mask = mask;
    cudaError_t e = launch_pred_mask(pp, pred->type, pred->op, di.sms, s);
    if (e != cudaSuccess) return cuda_status(e);
    e = launch_popc_blocks(pp.bs, di.sms, s);
    if (e != cudaSuccess) return cuda_status(e);
    return launch_writeout_3pass(col, l, hdr, r, true, pp.bs.item_flags, di, s);
}

int cs_workspace_check(void* d_ws, cs_stream_t stream)
{
    return check_workspace_error(d_ws, reinterpret_cast<cudaStream_t>(stream));
}

int compressstore_release(cs_stream_t stream)
{
    return release_cached_workspace(reinterpret_cast<cudaStream_t>(stream));
}

int compressstore_check(cs_stream_t stream)
{
    void* ws = nullptr;
    int st = lookup_cached_workspace(reinterpret_cast<cudaStream_t>(stream), &ws);
    if (st) return st;
    return check_workspace_error(ws, reinterpret_cast<cudaStream_t>(stream));
}

int cs_popc_chunks(const uint32_t* d_mask, uint64_t n, uint32_t chunk_length, uint32_t* d_chunk_counts,
                   cs_stream_t stream)
{
    if (!is_pow2(chunk_length) || chunk_length < 32 || chunk_length > 65536) return CS_ERR_INVALID_VALUE;
    if (n > MAX_N) return CS_ERR_NOT_SUPPORTED;
    if (n == 0) return CS_SUCCESS;
    if (!d_mask || !d_chunk_counts) return CS_ERR_INVALID_VALUE;
    if (!aligned(d_mask, 4) || !aligned(d_chunk_counts, 4)) return CS_ERR_MISALIGNED;
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    return cuda_status(launch_popc_chunks(d_mask, n, ilog2(chunk_length), d_chunk_counts, nullptr, nullptr, di.sms,
                                          reinterpret_cast<cudaStream_t>(stream)));
}

size_t cs_scan_workspace_size(uint64_t chunk_count)
{
    const uint64_t tiles = (chunk_count + SCAN_TILE - 1) / SCAN_TILE;
    return align256(sizeof(ws_header) + align256(8 * tiles));
}

int cs_chunk_prefix_sum(const uint32_t* d_chunk_counts, uint64_t chunk_count, uint64_t* d_chunk_offsets,
                        uint64_t* d_total, void* d_ws, size_t ws_bytes, cs_stream_t stream)
{
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (chunk_count == 0) {
        if (d_total) return cuda_status(cudaMemsetAsync(d_total, 0, sizeof(uint64_t), s));
        return CS_SUCCESS;
    }
    if (!d_chunk_counts || !d_chunk_offsets) return CS_ERR_INVALID_VALUE;
    if (!aligned(d_chunk_counts, 4) || !aligned(d_chunk_offsets, 8) || (d_total && !aligned(d_total, 8)))
        return CS_ERR_MISALIGNED;
    if (!d_ws || ws_bytes < cs_scan_workspace_size(chunk_count) || !aligned(d_ws, 256)) return CS_ERR_WORKSPACE;
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    uint8_t* ws = static_cast<uint8_t*>(d_ws);
    ScanParams sp{};
    sp.counts = d_chunk_counts;
    sp.count = chunk_count;
    sp.offsets = d_chunk_offsets;
    sp.total = d_total;
    sp.hdr = reinterpret_cast<ws_header*>(ws);
    sp.status = reinterpret_cast<uint64_t*>(ws + sizeof(ws_header));
    sp.num_tiles = (chunk_count + SCAN_TILE - 1) / SCAN_TILE;
    sp.timeout_ns = DEFAULT_TIMEOUT_NS;
    return cuda_status(launch_scan(sp, di.sms, s));
}

int cs_writeout(const void* d_in, const uint32_t* d_mask, void* d_out, uint64_t n, uint32_t elem_bytes,
                const uint64_t* d_chunk_offsets, const uint32_t* d_chunk_counts, uint32_t chunk_length, int32_t algo,
                cs_stream_t stream)
{
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8) return CS_ERR_INVALID_VALUE;
    if (!is_pow2(chunk_length) || chunk_length < 32 || chunk_length > 65536) return CS_ERR_INVALID_VALUE;
    if (algo != CS_ALGO_3PASS && algo != CS_ALGO_NAIVE) return CS_ERR_INVALID_VALUE;
    if (n > MAX_N) return CS_ERR_NOT_SUPPORTED;
    if (n == 0) return CS_SUCCESS;
    if (!d_in || !d_mask || !d_out || !d_chunk_offsets) return CS_ERR_INVALID_VALUE;
    if (!aligned(d_in, elem_bytes) || !aligned(d_out, elem_bytes) || !aligned(d_mask, 4) ||
        !aligned(d_chunk_offsets, 8))
        return CS_ERR_MISALIGNED;
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint32_t log2L = ilog2(chunk_length);
    const uint64_t ue = unit_elems_for(elem_bytes);
    if (algo == CS_ALGO_3PASS) {
        if (!(aligned(d_in, 16) && aligned(d_out, 16) && aligned(d_mask, 16))) return CS_ERR_MISALIGNED;
        if (chunk_length > ue) return CS_ERR_NOT_SUPPORTED;
        CompactParams p{};
        p.col0 = make_column(d_in, d_mask, d_out, n, elem_bytes, nullptr, const_cast<uint64_t*>(d_chunk_offsets));
        p.num_tiles = (n + ue - 1) / ue;
        p.hdr = nullptr; // no workspace: errors are not recorded, inconsistent offsets still never write
        p.chunk_log2 = log2L;
        p.skip = 1;
        p.timeout_ns = DEFAULT_TIMEOUT_NS;
        const uint32_t grid = persistent_grid(elem_bytes, 1, di, p.num_tiles, 0);
        return cuda_status(launch_compact_tma(p, elem_bytes, 1, grid, s));
    }
    return cuda_status(launch_writeout_naive(d_in, d_mask, d_out, n, elem_bytes, d_chunk_offsets, d_chunk_counts, log2L,
                                             nullptr, di.sms, s));
}

int cs_gen_payload(void* d_out, uint64_t n, uint32_t elem_bytes, uint64_t seed, int32_t float_unit, cs_stream_t stream)
{
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8) return CS_ERR_INVALID_VALUE;
    if (n == 0) return CS_SUCCESS;
    if (!d_out) return CS_ERR_INVALID_VALUE;
    if (!aligned(d_out, elem_bytes)) return CS_ERR_MISALIGNED;
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    return cuda_status(
        launch_gen_payload(d_out, n, elem_bytes, seed, float_unit, di.sms, reinterpret_cast<cudaStream_t>(stream)));
}

int cs_gen_mask_bernoulli(uint32_t* d_mask, uint64_t n, double p, uint64_t seed, cs_stream_t stream)
{
    if (n == 0) return CS_SUCCESS;
    if (!d_mask || !(p >= 0.0 && p <= 1.0)) return CS_ERR_INVALID_VALUE;
    if (!aligned(d_mask, 4)) return CS_ERR_MISALIGNED;
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    const uint64_t thr = (p >= 1.0) ? (1ull << 32) : static_cast<uint64_t>(p * 4294967296.0);
    return cuda_status(launch_gen_mask_bernoulli(d_mask, n, thr, seed, di.sms, reinterpret_cast<cudaStream_t>(stream)));
}

size_t cs_gen_mask_runs_workspace_size(uint64_t n)
{
    const uint64_t nw = (n + 31) / 32;
    return cs_scan_workspace_size(nw) + align256(4 * nw) + align256(8 * nw);
}

int cs_gen_mask_runs(uint32_t* d_mask, uint64_t n, double mean_run, uint64_t seed, void* d_ws, size_t ws_bytes,
                     cs_stream_t stream)
{
    if (n == 0) return CS_SUCCESS;
    if (!d_mask || !(mean_run >= 1.0)) return CS_ERR_INVALID_VALUE;
    if (!aligned(d_mask, 4)) return CS_ERR_MISALIGNED;
    if (!d_ws || ws_bytes < cs_gen_mask_runs_workspace_size(n) || !aligned(d_ws, 256)) return CS_ERR_WORKSPACE;
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint64_t nw = (n + 31) / 32;
    const uint64_t thr = static_cast<uint64_t>(4294967296.0 / mean_run);
    uint8_t* ws = static_cast<uint8_t*>(d_ws);
    const size_t scan_bytes = cs_scan_workspace_size(nw);
    uint32_t* counts = reinterpret_cast<uint32_t*>(ws + scan_bytes);
    uint64_t* offsets = reinterpret_cast<uint64_t*>(ws + scan_bytes + align256(4 * nw));
    cudaError_t e = launch_gen_runs_toggle(d_mask, counts, n, thr, seed, di.sms, s);
    if (e != cudaSuccess) return cuda_status(e);
    ScanParams sp{};
    sp.counts = counts;
    sp.count = nw;
    sp.offsets = offsets;
    sp.total = nullptr;
    sp.hdr = reinterpret_cast<ws_header*>(ws);
    sp.status = reinterpret_cast<uint64_t*>(ws + sizeof(ws_header));
    sp.num_tiles = (nw + SCAN_TILE - 1) / SCAN_TILE;
    sp.timeout_ns = DEFAULT_TIMEOUT_NS;
    sp.keep_begin = scan_bytes;
    sp.keep_end = scan_bytes + align256(4 * nw) + 8 * nw;
    e = launch_scan(sp, di.sms, s);
    if (e != cudaSuccess) return cuda_status(e);
    return cuda_status(launch_gen_runs_apply(d_mask, offsets, n, di.sms, s));
}

int cs_gen_mask_dense_prefix(uint32_t* d_mask, uint64_t n, float frac, cs_stream_t stream)
{
    if (n == 0) return CS_SUCCESS;
    if (!d_mask || !(frac >= 0.0f)) return CS_ERR_INVALID_VALUE;
    if (!aligned(d_mask, 4)) return CS_ERR_MISALIGNED;
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    uint64_t k = static_cast<uint64_t>(frac * static_cast<float>(n));
    if (k > n) k = n;
    return cuda_status(launch_gen_mask_dense_prefix(d_mask, n, k, di.sms, reinterpret_cast<cudaStream_t>(stream)));
}

int cs_gen_mask_pattern(uint32_t* d_mask, uint64_t n, uint32_t pattern, uint32_t pattern_length, cs_stream_t stream)
{
    if (pattern_length < 1 || pattern_length > 32) return CS_ERR_INVALID_VALUE;
    if (n == 0) return CS_SUCCESS;
    if (!d_mask) return CS_ERR_INVALID_VALUE;
    if (!aligned(d_mask, 4)) return CS_ERR_MISALIGNED;
    DeviceInfo di;
    int st = current_device_info(&di);
    if (st) return st;
    const uint32_t pm = pattern_length >= 32 ? pattern : (pattern & ((1u << pattern_length) - 1u));
    return cuda_status(
        launch_gen_mask_pattern(d_mask, n, pm, pattern_length, di.sms, reinterpret_cast<cudaStream_t>(stream)));
}

const char* cs_status_string(int status)
{
    switch (status) {
        case CS_PENDING: return "pending";
        case CS_SUCCESS: return "success";
        case CS_ERR_INVALID_VALUE: return "invalid value";
        case CS_ERR_MISALIGNED: return "misaligned pointer";
        case CS_ERR_WORKSPACE: return "workspace missing, too small or misaligned";
        case CS_ERR_CUDA: return "CUDA runtime error";
        case CS_ERR_TIMEOUT: return "bounded device wait timed out";
        case CS_ERR_NO_DEVICE: return "no usable sm_100 device";
        case CS_ERR_OUT_OF_MEMORY: return "out of device memory";
        case CS_ERR_NOT_SUPPORTED: return "not supported";
        case CS_ERR_ADMISSION: return "request exceeds the memory budget";
        default: return "unknown status";
    }
}

uint64_t cs_launch_count(void)
{
    return g_launches.load(std::memory_order_relaxed);
}

uint32_t cs_tile_elems(uint32_t elem_bytes)
{
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8) return 0;
    return tile_elems_for(elem_bytes);
}

uint32_t cs_compact_smem_bytes(uint32_t elem_bytes, int32_t algo)
{
    if (algo != CS_ALGO_1PASS && algo != CS_ALGO_3PASS) return 0;
    if (algo == CS_ALGO_3PASS) return compact_tma_smem_bytes(elem_bytes, 1);
    const uint32_t a = compact_tma_smem_bytes(elem_bytes, 0), b = compact_tma_smem_bytes(elem_bytes, 2);
    return a > b ? a : b; // the largest a 1-pass call may launch
}

uint32_t cs_version(void)
{
    return 0x000100u;
}

} // extern "C"
