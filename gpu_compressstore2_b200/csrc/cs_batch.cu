// cs_batch.cu — the batched form: a plan over many columns of uneven length and width.
//
// Every column runs the 3-pass hybrid with 4096-element chunks, but each pass is ONE launch
// for the whole batch: the fused popcount+scan kernel walks a flat list of all columns'
// 256K-element tiles (decoupled look-back confined to each column), the sparse-gather kernel
// walks all columns' 16K-element items, and one persistent TMA-staged writeout per element
// width walks all that width's 128 KB units round robin over every SM. Work-to-column maps
// and column descriptors are built on the host once (cs_plan.cu) and uploaded with the plan,
// so a unit finds its column with one load. The launches can be captured in a CUDA graph.
#include <vector>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"
#include "cs_plan.h"

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
    uint64_t timeout_ns = 2000000000ull;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t kernels_per_run = 0;
};

namespace {

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
    return plan_launch(b->dev, b->counts, b->grid, b->sms, b->timeout_ns, s);
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

    std::vector<ColumnDesc> desc;
    std::vector<uint64_t> chunk_base;
    int st = plan_columns(cols, ncols, desc, chunk_base, b->counts, &b->empty_counts);
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
    for (int wi = 0; wi < 4; ++wi) b->grid[wi] = plan_grid(1u << wi, b->counts.units[wi], b->sms);
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
