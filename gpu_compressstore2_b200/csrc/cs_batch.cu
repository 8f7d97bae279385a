// cs_batch.cu — the batched form: a plan over many columns of uneven length and width.
//
// Each column takes the 3-pass hybrid (4096-element chunks) or the 1-pass form, as the
// batch table of the autotuner says for its (width, size, selectivity) bucket; each pass is
// ONE launch for all the columns that take it: the reduce-then-scan popcount + prefix kernel
// walks a flat list of the 3-pass columns' 2^18-element blocks, the sparse-gather kernel walks
// their 16K-element items, one persistent TMA-staged writeout per element width walks that
// width's 128 KB units over every SM, and one 1-pass kernel per width walks the 1-pass
// columns' units (decoupled look-back confined to each column). Work-to-column maps and column
// descriptors are built on the host once (cs_plan.cu) and uploaded with the plan, so a unit
// finds its column with one load. The launches can be captured in a CUDA graph.
//
// Selectivity is measured when the plan is built (CS_ALGO_AUTO, and only when the table has a
// 1-pass entry): one popcount pass over the masks into plan-owned count words. The choice
// changes speed, never results, so masks that change between runs stay correct.
#include <vector>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"
#include "cs_plan.h"
#include "cs_tuning.h"

using namespace cs;

struct cs_batch {
    int device = 0;
    int sms = 0;
    std::vector<uint64_t*> empty_counts; // d_count of n == 0 columns
    void* dmem = nullptr;
    PlanLayout layout;
    PlanDevice dev;
    PlanCounts counts;
    uint32_t grid[4] = {0, 0, 0, 0};
    uint32_t grid1[4] = {0, 0, 0, 0};
    uint32_t one_pass_cols = 0;
    std::vector<cs_column> cols; // for the per-call loop
    uint64_t timeout_ns = 2000000000ull;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t kernels_per_run = 0;
};

namespace {

// Least payload the 3-pass columns of a mixed plan must hold to keep their form (about the
// bytes HBM moves in the 40 us their extra launches take).
constexpr uint64_t PLAN_3PASS_MIN_BYTES = 256ull << 20;

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
    return plan_launch(b->dev, b->counts, b->grid, b->sms, b->timeout_ns, s, b->grid1);
}

// Selected fraction of every column, from one reduce-then-scan popcount pass over the masks
// (into count words of a temporary plan, so nothing of the caller's is written).
int measure_selectivity(const cs_column* cols, uint32_t ncols, int sms, cudaStream_t s, std::vector<double>& sel)
{
    sel.assign(ncols, 0.0);
    std::vector<ColumnDesc> desc;
    std::vector<uint64_t> chunk_base;
    PlanCounts c;
    int st = plan_columns(cols, ncols, desc, chunk_base, c, nullptr);
    if (st != CS_SUCCESS) return st;
    if (!c.tiles) return CS_SUCCESS;
    const PlanLayout L = plan_layout(c, true);
    void* mem = nullptr;
    if (cudaMalloc(&mem, L.total) != cudaSuccess) {
        cudaGetLastError();
        return CS_ERR_OUT_OF_MEMORY;
    }
    const PlanMaps m = plan_maps(c);
    const PlanDevice d = plan_device(static_cast<uint8_t*>(mem), L, m);
    for (uint32_t i = 0; i < ncols; ++i) desc[i].d_count = d.counts + i;
    std::vector<uint8_t> img(m.bytes);
    plan_write_image(img.data(), m, d, desc, chunk_base);
    std::vector<uint64_t> counts(ncols, 0);
    cudaError_t e = launch_ws_init(d.hdr, L.total, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d.maps, img.data(), img.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) {
        BlockScanParams bp{};
        bp.cols = d.cols;
        bp.blk_col = d.tile_col;
        bp.num_blocks = c.tiles;
        bp.blk_sum = d.blk_sum;
        bp.blk_base = d.blk_base;
        bp.hdr = d.hdr;
        bp.chunk_log2 = 12;
        bp.keep_begin = d.keep_begin;
        bp.keep_end = d.keep_end;
        e = launch_popc_blocks(bp, sms, s);
    }
    if (e == cudaSuccess && ncols) e = cudaMemcpyAsync(counts.data(), d.counts, 8 * ncols, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(mem);
    if (e != cudaSuccess) return to_status(e);
    for (uint32_t i = 0; i < ncols; ++i)
        if (cols[i].n) sel[i] = static_cast<double>(counts[i]) / static_cast<double>(cols[i].n);
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
    int major = 0;
    if (cudaGetDevice(&b->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess ||
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, b->device) != cudaSuccess || major != 10) {
        delete b;
        return CS_ERR_NO_DEVICE;
    }
    if (cfg && cfg->timeout_ns) b->timeout_ns = cfg->timeout_ns;
    const int algo = cfg ? cfg->algo : CS_ALGO_AUTO;
    if (algo != CS_ALGO_AUTO && algo != CS_ALGO_1PASS && algo != CS_ALGO_3PASS) {
        delete b;
        return CS_ERR_INVALID_VALUE;
    }
    b->cols.assign(cols, cols + ncols);

    // per column: 1-pass or 3-pass (forced by cfg->algo, else the batch table's bucket)
    std::vector<uint8_t> one_pass(ncols, algo == CS_ALGO_1PASS ? 1 : 0);
    if (algo == CS_ALGO_AUTO && tune_batch_any_1pass()) {
        std::vector<double> sel;
        const int st = measure_selectivity(cols, ncols, b->sms, s, sel);
        if (st != CS_SUCCESS) {
            delete b;
            return st;
        }
        for (uint32_t i = 0; i < ncols; ++i)
            one_pass[i] = cols[i].n && tune_batch_lookup(cols[i].n, cols[i].elem_bytes, sel[i]) == CS_ALGO_1PASS;
        // Beside 1-pass columns, the 3-pass ones add a chain of their own (pass 1+2, the
        // sparse gather, a writeout per width: about 40 us of launches that wait on one
        // another on B200), and what their form saves is at most their payload reads. Below
        // PLAN_3PASS_MIN_BYTES of 3-pass payload they join the 1-pass kernels (batch256:
        // 0.602 -> 0.571 ms per replay with its six sparse columns moved).
        uint64_t bytes3 = 0, bytes1 = 0;
        for (uint32_t i = 0; i < ncols; ++i)
            (one_pass[i] ? bytes1 : bytes3) += cols[i].n * static_cast<uint64_t>(cols[i].elem_bytes);
        if (bytes1 && bytes3 < PLAN_3PASS_MIN_BYTES)
            for (uint32_t i = 0; i < ncols; ++i) one_pass[i] = cols[i].n ? 1 : 0;
    }
    for (uint32_t i = 0; i < ncols; ++i) b->one_pass_cols += one_pass[i] && cols[i].n ? 1u : 0u;

    std::vector<ColumnDesc> desc;
    std::vector<uint64_t> chunk_base;
    int st = plan_columns(cols, ncols, desc, chunk_base, b->counts, &b->empty_counts, &one_pass);
    if (st != CS_SUCCESS) {
        delete b;
        return st;
    }
    b->layout = plan_layout(b->counts, false);
    cudaError_t e = cudaMalloc(&b->dmem, b->layout.total);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete b;
        return CS_ERR_OUT_OF_MEMORY;
    }
    const PlanMaps maps = plan_maps(b->counts);
    b->dev = plan_device(static_cast<uint8_t*>(b->dmem), b->layout, maps);
    std::vector<uint8_t> img(maps.bytes);
    plan_write_image(img.data(), maps, b->dev, desc, chunk_base);
    e = launch_ws_init(b->dev.hdr, b->layout.total, s); // zeroes everything, writes the header
    if (e == cudaSuccess && !img.empty())
        e = cudaMemcpyAsync(b->dev.maps, img.data(), img.size(), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        cudaFree(b->dmem);
        delete b;
        return to_status(e);
    }
    // persistent grids (also applies the kernels' shared-memory attribute outside any capture)
    for (int wi = 0; wi < 4; ++wi) {
        b->grid[wi] = plan_grid(1u << wi, b->counts.units[wi], b->sms, 1);
        b->grid1[wi] = plan_grid(1u << wi, b->counts.units1[wi], b->sms, 0);
    }
    b->kernels_per_run = plan_kernels(b->counts);
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
    return cs_workspace_check(b->dev.hdr, stream);
}

int cs_batch_run_per_call(cs_batch* b, cs_stream_t stream)
{
    if (!b) return CS_ERR_INVALID_VALUE;
    for (const cs_column& c : b->cols) {
        const int st = compressstore(c.d_in, c.d_mask, c.d_out, c.n, c.elem_bytes, c.d_count, stream);
        if (st != CS_SUCCESS) return st;
    }
    return CS_SUCCESS;
}

uint32_t cs_batch_one_pass_columns(const cs_batch* b)
{
    return b ? b->one_pass_cols : 0u;
}

uint64_t cs_batch_device_bytes(const cs_batch* b)
{
    return b ? b->layout.total : 0;
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
