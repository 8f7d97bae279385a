// cs_plan.cu — the multi-column plan builder shared by the batched form and the serving
// loop (layout and launch order in cs_plan.h).
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"
#include "cs_plan.h"

namespace cs {

namespace {

constexpr uint64_t PLAN_MAX_N = (1ull << 40) - 1;

inline size_t a256(size_t x)
{
    return (x + 255) & ~static_cast<size_t>(255);
}

inline size_t a16(size_t x)
{
    return (x + 15) & ~static_cast<size_t>(15);
}

inline bool aligned_to(const void* p, uintptr_t a)
{
    return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0;
}

inline int to_status(cudaError_t e)
{
    if (e == cudaSuccess) return CS_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return CS_ERR_OUT_OF_MEMORY;
    return CS_ERR_CUDA;
}

constexpr uint64_t FUSED_TILE_ELEMS = 4096ull * FUSED_TILE_CHUNKS;
constexpr uint64_t SPARSE_ITEM_ELEMS = 16384ull;

} // namespace

void plan_column_work(uint64_t n, uint32_t w, uint64_t* tiles, uint64_t* items, uint64_t* units, uint64_t* chunks)
{
    const uint64_t ch = (n + 4095) / 4096;
    const uint64_t ue = unit_elems_for(w);
    *chunks = ch;
    *tiles = (ch + FUSED_TILE_CHUNKS - 1) / FUSED_TILE_CHUNKS;
    *items = sparse_items_for(n);
    *units = (n + ue - 1) / ue;
}

PlanCounts plan_capacity(uint64_t max_elems, uint32_t max_cols)
{
    // sum over columns of ceil(n_c / k) <= sum(n_c) / k + (number of columns)
    PlanCounts c;
    c.cols = max_cols;
    c.tiles = max_elems / FUSED_TILE_ELEMS + max_cols;
    c.items = max_elems / SPARSE_ITEM_ELEMS + max_cols;
    for (int wi = 0; wi < 4; ++wi) c.units[wi] = max_elems / unit_elems_for(1u << wi) + max_cols;
    c.chunks = max_elems / 4096 + max_cols;
    return c;
}

PlanMaps plan_maps(const PlanCounts& c)
{
    PlanMaps m;
    size_t off = 0;
    m.off_cols = off;
    off += a16(sizeof(ColumnDesc) * c.cols);
    m.off_tile = off;
    off += a16(4 * c.tiles);
    m.off_item = off;
    off += a16(4 * c.items);
    for (int wi = 0; wi < 4; ++wi) {
        m.off_unit[wi] = off;
        off += a16(4 * c.units[wi]);
    }
    for (int wi = 0; wi < 4; ++wi) {
        m.off_unit1[wi] = off;
        off += a16(4 * c.units1[wi]);
    }
    m.bytes = off;
    return m;
}

PlanLayout plan_layout(const PlanCounts& caps, bool with_counts)
{
    PlanLayout L;
    size_t off = sizeof(ws_header);
    L.off_counts = off;
    if (with_counts) off += a256(8 * caps.cols);
    L.off_maps = off;
    L.maps_bytes = plan_maps(caps).bytes;
    off += a256(L.maps_bytes);
    L.off_offsets = off;
    off += a256(8 * caps.chunks);
    L.off_blk_base = off;
    off += a256(8 * caps.tiles);
    L.off_item_flags = off;
    off += a256(4 * caps.items);
    L.off_blk_sum = off;
    off += a256(8 * caps.tiles);
    L.off_flags = off;
    off += a256(4 * POPC_FLAG_SLOTS);
    L.off_status = off;
    uint64_t st = 0;
    for (int wi = 0; wi < 4; ++wi) {
        L.status_base[wi] = st;
        st += caps.units1[wi];
    }
    off += a256(8 * st);
    L.total = a256(off);
    return L;
}

PlanDevice plan_device(uint8_t* base, const PlanLayout& L, const PlanMaps& m)
{
    PlanDevice d;
    d.hdr = reinterpret_cast<ws_header*>(base);
    d.blk_sum = reinterpret_cast<uint64_t*>(base + L.off_blk_sum);
    d.blk_base = reinterpret_cast<uint64_t*>(base + L.off_blk_base);
    d.item_flags = reinterpret_cast<uint32_t*>(base + L.off_item_flags);
    d.flags = reinterpret_cast<uint32_t*>(base + L.off_flags);
    d.maps = base + L.off_maps;
    d.cols = reinterpret_cast<ColumnDesc*>(d.maps + m.off_cols);
    d.tile_col = reinterpret_cast<uint32_t*>(d.maps + m.off_tile);
    d.item_col = reinterpret_cast<uint32_t*>(d.maps + m.off_item);
    for (int wi = 0; wi < 4; ++wi) {
        d.unit_col[wi] = reinterpret_cast<uint32_t*>(d.maps + m.off_unit[wi]);
        d.unit1_col[wi] = reinterpret_cast<uint32_t*>(d.maps + m.off_unit1[wi]);
        d.status[wi] = reinterpret_cast<uint64_t*>(base + L.off_status) + L.status_base[wi];
    }
    d.offsets = reinterpret_cast<uint64_t*>(base + L.off_offsets);
    d.counts = reinterpret_cast<uint64_t*>(base + L.off_counts);
    d.keep_begin = L.off_counts;
    d.keep_end = L.off_blk_sum;
    d.total = L.total;
    return d;
}

int plan_columns(const cs_column* cols, uint32_t ncols, std::vector<ColumnDesc>& desc,
                 std::vector<uint64_t>& chunk_base, PlanCounts& tot, std::vector<uint64_t*>* empty,
                 const std::vector<uint8_t>* one_pass)
{
    desc.assign(ncols, ColumnDesc{});
    chunk_base.assign(ncols, 0);
    tot = PlanCounts{};
    tot.cols = ncols;
    for (uint32_t c = 0; c < ncols; ++c) {
        const cs_column& col = cols[c];
        const uint32_t w = col.elem_bytes;
        if (w != 1 && w != 2 && w != 4 && w != 8) return CS_ERR_INVALID_VALUE;
        if (!col.d_count) return CS_ERR_INVALID_VALUE;
        if (col.n > PLAN_MAX_N) return CS_ERR_NOT_SUPPORTED;
        if (!aligned_to(col.d_count, 8)) return CS_ERR_MISALIGNED;
        ColumnDesc& d = desc[c];
        d.elem_bytes = w;
        d.d_count = col.d_count;
        if (col.n == 0) {
            if (empty) empty->push_back(col.d_count);
            continue;
        }
        if (!col.d_in || !col.d_mask || !col.d_out) return CS_ERR_INVALID_VALUE;
        if (!aligned_to(col.d_in, 16) || !aligned_to(col.d_out, 16) || !aligned_to(col.d_mask, 16))
            return CS_ERR_MISALIGNED;
        d.in = static_cast<const uint8_t*>(col.d_in);
        d.mask = static_cast<const uint32_t*>(col.d_mask);
        d.out = static_cast<uint8_t*>(col.d_out);
        d.n = col.n;
        uint64_t tiles, items, units, chunks;
        plan_column_work(col.n, w, &tiles, &items, &units, &chunks);
        const int wi = plan_width_index(w);
        if (one_pass && (*one_pass)[c]) {
            d.one_pass = 1;
            d.unit_base = tot.units1[wi];
            tot.units1[wi] += units;
            continue;
        }
        d.tile_base = tot.tiles;
        d.item_base = tot.items;
        d.unit_base = tot.units[wi];
        chunk_base[c] = tot.chunks;
        tot.tiles += tiles;
        tot.items += items;
        tot.units[wi] += units;
        tot.chunks += chunks;
    }
    if (tot.tiles > 0xffffffffull || tot.items > 0xffffffffull) return CS_ERR_NOT_SUPPORTED;
    return CS_SUCCESS;
}

void plan_write_image(uint8_t* img, const PlanMaps& m, const PlanDevice& dev, const std::vector<ColumnDesc>& desc,
                      const std::vector<uint64_t>& chunk_base)
{
    std::memset(img, 0, m.bytes);
    ColumnDesc* hcols = reinterpret_cast<ColumnDesc*>(img + m.off_cols);
    uint32_t* htile = reinterpret_cast<uint32_t*>(img + m.off_tile);
    uint32_t* hitem = reinterpret_cast<uint32_t*>(img + m.off_item);
    uint32_t* hunit[4];
    for (int wi = 0; wi < 4; ++wi) hunit[wi] = reinterpret_cast<uint32_t*>(img + m.off_unit[wi]);
    for (uint32_t c = 0; c < desc.size(); ++c) {
        ColumnDesc d = desc[c];
        if (d.n && d.one_pass) {
            uint64_t tiles, items, units, chunks;
            plan_column_work(d.n, d.elem_bytes, &tiles, &items, &units, &chunks);
            uint32_t* hu1 = reinterpret_cast<uint32_t*>(img + m.off_unit1[plan_width_index(d.elem_bytes)]);
            for (uint64_t u = 0; u < units; ++u) hu1[d.unit_base + u] = c;
        } else if (d.n) {
            d.offsets = dev.offsets + chunk_base[c];
            d.blk_base = dev.blk_base + d.tile_base;
            uint64_t tiles, items, units, chunks;
            plan_column_work(d.n, d.elem_bytes, &tiles, &items, &units, &chunks);
            for (uint64_t t = 0; t < tiles; ++t) htile[d.tile_base + t] = c;
            for (uint64_t t = 0; t < items; ++t) hitem[d.item_base + t] = c;
            uint32_t* hu = hunit[plan_width_index(d.elem_bytes)];
            for (uint64_t u = 0; u < units; ++u) hu[d.unit_base + u] = c;
        }
        hcols[c] = d;
    }
}

uint32_t plan_grid(uint32_t w, uint64_t units, int sms, int mode)
{
    if (!units) return 0;
    int bps = compact_tma_blocks_per_sm(w, mode);
    if (bps < 1) bps = 1;
    uint64_t g = static_cast<uint64_t>(bps) * sms;
    if (g > units) g = units;
    return static_cast<uint32_t>(g ? g : 1);
}

uint32_t plan_kernels(const PlanCounts& c)
{
    uint32_t k = (c.tiles ? 1u : 0u) + (c.items ? 1u : 0u);
    for (int wi = 0; wi < 4; ++wi) k += (c.units[wi] ? 1u : 0u) + (c.units1[wi] ? 1u : 0u);
    return k;
}

int plan_launch(const PlanDevice& d, const PlanCounts& c, const uint32_t grid[4], int sms, uint64_t timeout_ns,
                cudaStream_t s, const uint32_t* grid1)
{
    if (c.tiles) {
        BlockScanParams bp{};
        bp.cols = d.cols;
        bp.blk_col = d.tile_col;
        bp.num_blocks = c.tiles;
        bp.blk_sum = d.blk_sum;
        bp.blk_base = d.blk_base;
        bp.hdr = d.hdr;
        bp.item_flags = d.item_flags;
        bp.chunk_log2 = 12;
        bp.keep_begin = d.keep_begin;
        bp.keep_end = d.keep_end;
        cudaError_t e = launch_popc_blocks(bp, sms, s);
        if (e != cudaSuccess) return to_status(e);
    }
    if (c.items) {
        SparseParams spp{};
        spp.cols = d.cols;
        spp.item_col = d.item_col;
        spp.num_items = c.items;
        spp.hdr = d.hdr;
        spp.chunk_log2 = 12;
        spp.item_flags = d.item_flags;
        cudaError_t e = launch_writeout_sparse(spp, sms, s);
        if (e != cudaSuccess) return to_status(e);
    }
    for (int wi = 0; wi < 4; ++wi) {
        if (!c.units[wi]) continue;
        const uint32_t w = 1u << wi;
        CompactParams p{};
        p.num_tiles = c.units[wi];
        p.hdr = d.hdr;
        p.sparse_max = unit_elems_for(w) / 32;
        p.chunk_log2 = 12;
        p.skip = 1;
        p.timeout_ns = timeout_ns;
        p.cols = d.cols;
        p.unit_col = d.unit_col[wi];
        cudaError_t e = launch_compact_tma(p, w, 1, grid[wi], s);
        if (e != cudaSuccess) return to_status(e);
    }
    for (int wi = 0; wi < 4; ++wi) {
        if (!c.units1[wi]) continue;
        if (!grid1) return CS_ERR_INVALID_VALUE;
        const uint32_t w = 1u << wi;
        CompactParams p{};
        p.num_tiles = c.units1[wi];
        p.hdr = d.hdr;
        p.status = d.status[wi];
        p.skip = 1;
        p.timeout_ns = timeout_ns;
        p.cols = d.cols;
        p.unit_col = d.unit1_col[wi];
        p.keep_begin = d.keep_begin;
        p.keep_end = d.keep_end;
        // a width with many 1-pass units takes the deeper payload ring, as the plain call does
        // for long columns (batch256: +0.4%)
        const int mode = (w >= 4 && c.units1[wi] >= 16ull * grid1[wi]) ? 2 : 0;
        cudaError_t e = launch_compact_tma(p, w, mode, grid1[wi], s);
        if (e != cudaSuccess) return to_status(e);
    }
    return CS_SUCCESS;
}

} // namespace cs
