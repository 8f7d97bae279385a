// cs_plan.h — building and launching a multi-column plan: the flat work lists (fused-scan
// tiles, sparse items, TMA units per width), their work-to-column maps and the column
// descriptors, laid out in one device buffer. Shared by the batched form (cs_batch.cu),
// which builds a plan once, and the serving loop (cs_server.cu), which rebuilds one per
// batch inside a slot buffer sized for a capacity.
//
// Buffer layout (offsets 256-byte aligned):
//   header | counts | maps | chunk offsets | block prefixes | item flags || block sums | pass-1 sparse flags
//   | 1-pass look-back statuses
// (a "tile" of the plan is a block of 2^18 elements of one column, the unit of the
// reduce-then-scan pass). The epoch-wrap clear zeroes everything after the header except
// [keep_begin, keep_end) = [counts, ||), so the per-column counts, the maps and the offsets
// and block prefixes the pass just wrote survive a wrap. Counts sit right after the header so that the header's error word and every count
// come back to the host in ONE copy. The maps region holds, packed with 16-byte aligned
// sub-arrays, the column descriptors, tile->column, item->column and per-width unit->column
// maps of ONE plan; a slot sized for a capacity is rewritten with each batch's packed maps by
// a single host-to-device copy.
#pragma once
#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"

namespace cs {

struct PlanCounts {
    uint64_t tiles = 0;               // 2^18-element blocks (64 chunks of 4096) over the 3-pass columns
    uint64_t items = 0;               // sparse-kernel items (16K elements) over the 3-pass columns
    uint64_t units[4] = {0, 0, 0, 0}; // TMA units of the 3-pass columns per width index (1, 2, 4, 8 bytes)
    uint64_t units1[4] = {0, 0, 0, 0}; // TMA units of the 1-pass columns per width index
    uint64_t chunks = 0;              // 4096-element chunks over the 3-pass columns (offsets array)
    uint64_t cols = 0;
};

// Packed maps of one plan, offsets relative to the start of the maps region.
struct PlanMaps {
    size_t off_cols = 0, off_tile = 0, off_item = 0;
    size_t off_unit[4] = {0, 0, 0, 0};
    size_t off_unit1[4] = {0, 0, 0, 0};
    size_t bytes = 0;
};

struct PlanLayout {
    size_t off_counts = 0, off_maps = 0, maps_bytes = 0, off_offsets = 0, off_blk_base = 0, off_item_flags = 0;
    size_t off_blk_sum = 0, off_flags = 0, off_status = 0, total = 0;
    uint64_t status_base[4] = {0, 0, 0, 0}; // first look-back status of each width's 1-pass units
};

struct PlanDevice {
    ws_header* hdr = nullptr;
    uint64_t* blk_sum = nullptr;
    uint64_t* blk_base = nullptr;
    uint32_t* item_flags = nullptr; // sparse items marked by pass 1 (epoch tagged)
    uint32_t* flags = nullptr;
    uint8_t* maps = nullptr;
    ColumnDesc* cols = nullptr;
    uint32_t* tile_col = nullptr;
    uint32_t* item_col = nullptr;
    uint32_t* unit_col[4] = {nullptr, nullptr, nullptr, nullptr};
    uint32_t* unit1_col[4] = {nullptr, nullptr, nullptr, nullptr};
    uint64_t* status[4] = {nullptr, nullptr, nullptr, nullptr}; // look-back statuses of each width's 1-pass units
    uint64_t* offsets = nullptr;
    uint64_t* counts = nullptr; // per-column count words (present when the layout reserved them)
    size_t keep_begin = 0, keep_end = 0, total = 0;
};

inline int plan_width_index(uint32_t w)
{
    return w == 1 ? 0 : w == 2 ? 1 : w == 4 ? 2 : 3;
}

// Work of one column of n elements of width w.
void plan_column_work(uint64_t n, uint32_t w, uint64_t* tiles, uint64_t* items, uint64_t* units, uint64_t* chunks);

// Upper bound on the work of any set of at most `max_cols` columns holding at most
// `max_elems` elements in total, of any widths.
PlanCounts plan_capacity(uint64_t max_elems, uint32_t max_cols);

PlanMaps plan_maps(const PlanCounts& c);

// Layout of a buffer for a capacity; `with_counts` reserves one count word per column.
PlanLayout plan_layout(const PlanCounts& caps, bool with_counts);

// Device pointers of the plan whose packed maps are `m`, inside a buffer at dbase laid out as L.
PlanDevice plan_device(uint8_t* dbase, const PlanLayout& L, const PlanMaps& m);

// Validate columns, assign work bases and accumulate totals. Zero-length columns are listed
// in `empty` (their count must be written as 0). `one_pass` (may be null: every column 3-pass)
// marks the columns that take the 1-pass form: they get units in their width's 1-pass list and
// no blocks, items or chunks. Returns a cs_status.
int plan_columns(const cs_column* cols, uint32_t ncols, std::vector<ColumnDesc>& desc,
                 std::vector<uint64_t>& chunk_base, PlanCounts& tot, std::vector<uint64_t*>* empty,
                 const std::vector<uint8_t>* one_pass = nullptr);

// Write the descriptors and maps as the host image (m.bytes) of the maps region; each
// descriptor's offsets and block-prefix pointers refer to dev.offsets and dev.blk_base.
void plan_write_image(uint8_t* img, const PlanMaps& m, const PlanDevice& dev, const std::vector<ColumnDesc>& desc,
                      const std::vector<uint64_t>& chunk_base);

// Persistent grid of the TMA kernel (mode 1: 3-pass writeout, 0: 1-pass) for `units` units of width w.
uint32_t plan_grid(uint32_t w, uint64_t units, int sms, int mode = 1);

// Kernels one run of the plan launches.
uint32_t plan_kernels(const PlanCounts& c);

// Enqueue the plan's kernels on the stream: for the 3-pass columns the reduce-then-scan
// popcount + prefix pass, the sparse gather and one TMA writeout per width present; then one
// 1-pass TMA kernel per width with 1-pass columns (grid1, may be null when there are none).
// The 1-pass kernels come last: each advances the workspace epoch, which the 3-pass writeouts
// read to validate the pass-2 results. Returns a cs_status.
int plan_launch(const PlanDevice& d, const PlanCounts& c, const uint32_t grid[4], int sms, uint64_t timeout_ns,
                cudaStream_t s, const uint32_t* grid1 = nullptr);

} // namespace cs
