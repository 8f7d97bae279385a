// cs_batch.cu — the batched form: a plan over many columns of uneven length and width.
//
// Every column runs the 3-pass hybrid with 4096-element chunks, but each pass is ONE launch
// for the whole batch: the fused popcount+scan kernel walks a flat list of all columns'
// 1M-element tiles (decoupled look-back confined to each column), the sparse-gather kernel
// walks all columns' 16K-element items, and one persistent TMA-staged writeout per element
// width walks all that width's 128 KB units round robin over every SM. Work-to-column maps
// and column descriptors are built on the host once and uploaded with the plan, so a unit
// finds its column with one load. The launches can be captured in a CUDA graph.
#include <algorithm>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"

using namespace cs;

struct cs_batch {
    int device = 0;
    int sms = 0;
    uint32_t ncols = 0;
    std::vector<uint64_t*> empty_counts; // d_count of n == 0 columns
    void* dmem = nullptr;
    size_t dbytes = 0;
    ws_header* hdr = nullptr;
    uint64_t* status = nullptr;
    uint32_t* flags = nullptr;
    ColumnDesc* d_cols = nullptr;
    uint32_t* d_tile_col = nullptr;
    uint32_t* d_item_col = nullptr;
    uint32_t* d_unit_col[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t total_tiles = 0;
    uint64_t total_items = 0;
    uint64_t units[4] = {0, 0, 0, 0};
    uint32_t grid[4] = {0, 0, 0, 0};
    uint64_t timeout_ns = 2000000000ull;
    size_t keep_begin = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t kernels_per_run = 0;
};

namespace {

constexpr uint64_t MAX_N = (1ull << 40) - 1;

inline size_t a256(size_t x)
{
    return (x + 255) & ~static_cast<size_t>(255);
}

inline bool aligned_to(const void* p, uintptr_t a)
{
    return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0;
}

inline int wi_of(uint32_t w)
{
    return w == 1 ? 0 : w == 2 ? 1 : w == 4 ? 2 : 3;
}

inline int to_status(cudaError_t e)
{
    if (e == cudaSuccess) return CS_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return CS_ERR_OUT_OF_MEMORY;
    return CS_ERR_CUDA;
}

int run_direct(cs_batch* b, cudaStream_t s)
{
    for (uint64_t* c : b->empty_counts) {
        cudaError_t e = cudaMemsetAsync(c, 0, sizeof(uint64_t), s);
        if (e != cudaSuccess) return to_status(e);
    }
    if (b->total_tiles) {
        ScanParams sp{};
        sp.hdr = b->hdr;
        sp.status = b->status;
        sp.num_tiles = b->total_tiles;
        sp.timeout_ns = b->timeout_ns;
        sp.popc_cta_flags = b->flags;
        sp.popc_flags = b->flags;
        sp.keep_begin = b->keep_begin;
        sp.keep_end = b->dbytes;
        sp.cols = b->d_cols;
        sp.tile_col = b->d_tile_col;
        cudaError_t e = launch_popc_scan_4096(sp, b->sms, s);
        if (e != cudaSuccess) return to_status(e);
    }
    if (b->total_items) {
        SparseParams spp{};
        spp.cols = b->d_cols;
        spp.item_col = b->d_item_col;
        spp.num_items = b->total_items;
        spp.hdr = b->hdr;
        spp.chunk_log2 = 12;
        cudaError_t e = launch_writeout_sparse(spp, b->sms, s);
        if (e != cudaSuccess) return to_status(e);
    }
    for (int wi = 0; wi < 4; ++wi) {
        if (!b->units[wi]) continue;
        const uint32_t w = 1u << wi;
        CompactParams p{};
        p.num_tiles = b->units[wi];
        p.hdr = b->hdr;
        p.sparse_max = unit_elems_for(w) / 32;
        p.chunk_log2 = 12;
        p.skip = 1;
        p.timeout_ns = b->timeout_ns;
        p.cols = b->d_cols;
        p.unit_col = b->d_unit_col[wi];
        cudaError_t e = launch_compact_tma(p, w, 1, b->grid[wi], s);
        if (e != cudaSuccess) return to_status(e);
    }
    return CS_SUCCESS;
}

} // namespace

extern "C" {

int cs_batch_create(cs_batch** out, const cs_column* cols, uint32_t ncols, const cs_config* cfg, cs_stream_t stream)
{
    if (!out || (!cols && ncols)) return CS_ERR_INVALID_VALUE;
    *out = nullptr;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    auto b = new cs_batch();
    if (cudaGetDevice(&b->device) != cudaSuccess) {
        delete b;
        return CS_ERR_NO_DEVICE;
    }
    int major = 0;
    if (cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, b->device) != cudaSuccess || major != 10) {
        delete b;
        return CS_ERR_NO_DEVICE;
    }
    if (cfg && cfg->timeout_ns) b->timeout_ns = cfg->timeout_ns;
    b->ncols = ncols;

    // host-side plan
    std::vector<ColumnDesc> desc(ncols);
    std::vector<uint64_t> chunk_base(ncols, 0);
    uint64_t total_chunks = 0;
    for (uint32_t c = 0; c < ncols; ++c) {
        const cs_column& col = cols[c];
        const uint32_t w = col.elem_bytes;
        if (w != 1 && w != 2 && w != 4 && w != 8) {
            delete b;
            return CS_ERR_INVALID_VALUE;
        }
        if (!col.d_count) {
            delete b;
            return CS_ERR_INVALID_VALUE;
        }
        if (col.n > MAX_N) {
            delete b;
            return CS_ERR_NOT_SUPPORTED;
        }
        if (!aligned_to(col.d_count, 8)) {
            delete b;
            return CS_ERR_MISALIGNED;
        }
        ColumnDesc& d = desc[c];
        d.elem_bytes = w;
        d.d_count = col.d_count;
        if (col.n == 0) {
            b->empty_counts.push_back(col.d_count);
            continue;
        }
        if (!col.d_in || !col.d_mask || !col.d_out) {
            delete b;
            return CS_ERR_INVALID_VALUE;
        }
        if (!aligned_to(col.d_in, 16) || !aligned_to(col.d_out, 16) || !aligned_to(col.d_mask, 16)) {
            delete b;
            return CS_ERR_MISALIGNED;
        }
        d.in = static_cast<const uint8_t*>(col.d_in);
        d.mask = static_cast<const uint32_t*>(col.d_mask);
        d.out = static_cast<uint8_t*>(col.d_out);
        d.n = col.n;
        const uint64_t chunks = (col.n + 4095) / 4096;
        const uint64_t tiles = (chunks + FUSED_TILE_CHUNKS - 1) / FUSED_TILE_CHUNKS;
        const uint64_t items = sparse_items_for(col.n);
        const uint64_t ue = unit_elems_for(w);
        const uint64_t units = (col.n + ue - 1) / ue;
        d.tile_base = b->total_tiles;
        d.item_base = b->total_items;
        d.unit_base = b->units[wi_of(w)];
        chunk_base[c] = total_chunks;
        b->total_tiles += tiles;
        b->total_items += items;
        b->units[wi_of(w)] += units;
        total_chunks += chunks;
    }
    if (b->total_tiles > 0xffffffffull || b->total_items > 0xffffffffull) {
        delete b;
        return CS_ERR_NOT_SUPPORTED;
    }

    // device layout: header | statuses | flags || columns | maps | offsets  (|| = keep_begin)
    size_t off = sizeof(ws_header);
    const size_t off_status = off;
    off += a256(8 * b->total_tiles);
    const size_t off_flags = off;
    off += a256(4 * POPC_FLAG_SLOTS);
    b->keep_begin = off;
    const size_t off_cols = off;
    off += a256(sizeof(ColumnDesc) * ncols);
    const size_t off_tile = off;
    off += a256(4 * b->total_tiles);
    const size_t off_item = off;
    off += a256(4 * b->total_items);
    size_t off_unit[4];
    for (int wi = 0; wi < 4; ++wi) {
        off_unit[wi] = off;
        off += a256(4 * b->units[wi]);
    }
    const size_t off_offsets = off;
    off += a256(8 * total_chunks);
    b->dbytes = a256(off);

    cudaError_t e = cudaMalloc(&b->dmem, b->dbytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return CS_ERR_OUT_OF_MEMORY;
    }
    uint8_t* base = static_cast<uint8_t*>(b->dmem);
    b->hdr = reinterpret_cast<ws_header*>(base);
    b->status = reinterpret_cast<uint64_t*>(base + off_status);
    b->flags = reinterpret_cast<uint32_t*>(base + off_flags);
    b->d_cols = reinterpret_cast<ColumnDesc*>(base + off_cols);
    b->d_tile_col = reinterpret_cast<uint32_t*>(base + off_tile);
    b->d_item_col = reinterpret_cast<uint32_t*>(base + off_item);
    for (int wi = 0; wi < 4; ++wi) b->d_unit_col[wi] = reinterpret_cast<uint32_t*>(base + off_unit[wi]);
    uint64_t* d_offsets = reinterpret_cast<uint64_t*>(base + off_offsets);

    // host image of [keep_begin, off_offsets): descriptors and work-to-column maps
    std::vector<uint8_t> img(off_offsets - b->keep_begin, 0);
    ColumnDesc* hcols = reinterpret_cast<ColumnDesc*>(img.data() + (off_cols - b->keep_begin));
    uint32_t* htile = reinterpret_cast<uint32_t*>(img.data() + (off_tile - b->keep_begin));
    uint32_t* hitem = reinterpret_cast<uint32_t*>(img.data() + (off_item - b->keep_begin));
    uint32_t* hunit[4];
    for (int wi = 0; wi < 4; ++wi) hunit[wi] = reinterpret_cast<uint32_t*>(img.data() + (off_unit[wi] - b->keep_begin));
    for (uint32_t c = 0; c < ncols; ++c) {
        ColumnDesc d = desc[c];
        if (d.n) {
            d.offsets = d_offsets + chunk_base[c];
            const uint64_t chunks = (d.n + 4095) / 4096;
            const uint64_t tiles = (chunks + FUSED_TILE_CHUNKS - 1) / FUSED_TILE_CHUNKS;
            for (uint64_t t = 0; t < tiles; ++t) htile[d.tile_base + t] = c;
            for (uint64_t t = 0; t < sparse_items_for(d.n); ++t) hitem[d.item_base + t] = c;
            const uint64_t ue = unit_elems_for(d.elem_bytes);
            const uint64_t units = (d.n + ue - 1) / ue;
            for (uint64_t u = 0; u < units; ++u) hunit[wi_of(d.elem_bytes)][d.unit_base + u] = c;
        }
        hcols[c] = d;
    }
    e = launch_ws_init(b->hdr, b->dbytes, s); // zeroes everything, writes the header
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + b->keep_begin, img.data(), img.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaFree(b->dmem);
        delete b;
        return to_status(e);
    }
    // persistent grids (also applies the kernels' shared-memory attribute outside any capture)
    for (int wi = 0; wi < 4; ++wi) {
        if (!b->units[wi]) continue;
        int bps = compact_tma_blocks_per_sm(1u << wi, 1);
        if (bps < 1) bps = 1;
        uint64_t g = static_cast<uint64_t>(bps) * b->sms;
        if (g > b->units[wi]) g = b->units[wi];
        b->grid[wi] = static_cast<uint32_t>(g ? g : 1);
    }
    b->kernels_per_run = (b->total_tiles ? 1 : 0) + (b->total_items ? 1 : 0);
    for (int wi = 0; wi < 4; ++wi) b->kernels_per_run += b->units[wi] ? 1 : 0;
    *out = b;
    return CS_SUCCESS;
}

int cs_batch_run(cs_batch* b, cs_stream_t stream)
{
    if (!b) return CS_ERR_INVALID_VALUE;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (b->exec) {
        cudaError_t e = cudaGraphLaunch(b->exec, s);
        if (e == cudaSuccess) note_launch(b->kernels_per_run);
        return to_status(e);
    }
    return run_direct(b, s);
}

int cs_batch_graph(cs_batch* b, cs_stream_t stream)
{
    if (!b) return CS_ERR_INVALID_VALUE;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!s) return CS_ERR_INVALID_VALUE; // the legacy default stream cannot be captured
    if (b->exec) {
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    if (b->graph) {
        cudaGraphDestroy(b->graph);
        b->graph = nullptr;
    }
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return to_status(e);
    const uint64_t before = cs_launch_count();
    const int st = run_direct(b, s);
    cudaGraph_t g = nullptr;
    e = cudaStreamEndCapture(s, &g);
    note_launch(0 - (cs_launch_count() - before)); // captured, not executed
    if (st != CS_SUCCESS) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (e != cudaSuccess) return to_status(e);
    e = cudaGraphInstantiate(&b->exec, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return to_status(e);
    }
    b->graph = g;
    return CS_SUCCESS;
}

int cs_batch_check(cs_batch* b, cs_stream_t stream)
{
    if (!b) return CS_ERR_INVALID_VALUE;
    return cs_workspace_check(b->hdr, stream);
}

uint64_t cs_batch_device_bytes(const cs_batch* b)
{
    return b ? b->dbytes : 0;
}

uint32_t cs_batch_launches(const cs_batch* b)
{
    return b ? (b->exec ? 1u : b->kernels_per_run) : 0u;
}

int cs_batch_destroy(cs_batch* b)
{
    if (!b) return CS_SUCCESS;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (b->dmem) cudaFree(b->dmem);
    delete b;
    return CS_SUCCESS;
}

} // extern "C"
