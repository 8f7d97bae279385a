// cs_noalloc.cu — compressstore_noalloc: the plain compaction for callers that must not
// allocate device memory.
//
// Some callers cannot call cudaMalloc: code embedded in a host application (a database or
// dataframe engine, an inference server) whose device memory is entirely reserved and
// handed out by that application's own pool, or a latency-critical loop that cannot take
// the implicit synchronisation an allocation may cause. The plain compressstore keeps a
// scratch workspace that it grows with stream-ordered allocations, and compressstore_ex
// needs the caller to provide one. This entry point instead uses a fixed scratch area
// compiled into the library: a file-scope __device__ array that every GPU which loads the
// library holds until the process exits.
//
// The scratch is shared by every call on a device and keeps what the last call left in
// it. Nothing in it has to be cleared between calls: the look-back statuses carry the
// epoch of the call that wrote them, and the dynamic work counters are put back to zero by
// the last CTA of each kernel. It is zeroed when the first call on a device sets it up.
// Calls that overlap on the GPU (for example on two streams) race on that scratch and
// must not be made.
//
// The scratch layout depends on n, the element width and the chunk length. This entry point
// fixes the chunk length at 4096 elements, whatever the tuning table says, so the layout is
// bounded by n alone: at n = CS_NOALLOC_MAX_N it needs about 3.4 MB for every width (chunk
// counts and offsets 3 MB, look-back statuses at most 64 KB, the rest under 0.4 MB), inside
// CS_NOALLOC_SCRATCH_BYTES. The output does not depend on the chunk length.
//
// Every call re-reads the array's device address (cudaGetSymbolAddress is a lookup, not a
// stream operation). If it differs from the one set up before (the first call on a device,
// or after cudaDeviceReset reloaded the module), the array is zeroed again on `stream`
// before the call's kernels.
#include <mutex>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = CS_NOALLOC_SCRATCH_BYTES; // per device
constexpr uint64_t NOALLOC_MAX_N = CS_NOALLOC_MAX_N;
constexpr uint32_t NOALLOC_CHUNK = 4096; // fixed chunk length: bounds the layout (see above)
constexpr int NOALLOC_MAX_DEVICES = 64;

struct DeviceScratch {
    void* ptr = nullptr; // device address of the scratch array on that device
    bool ready = false;
};

std::mutex g_noalloc_mu;
DeviceScratch g_noalloc_dev[NOALLOC_MAX_DEVICES];

} // namespace

// The scratch. In host code this name is only a handle: its device address comes from
// cudaGetSymbolAddress, taken with the device current.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

extern "C" {

int compressstore_noalloc(const void* d_in, const void* d_mask, void* d_out, uint64_t n, uint32_t elem_bytes,
                          uint64_t* d_count, cs_stream_t stream)
{
    if (n > NOALLOC_MAX_N) return CS_ERR_NOT_SUPPORTED; // larger columns need compressstore / _ex
    cs_config cfg{};
    cfg.algo = CS_ALGO_AUTO;
    cfg.chunk_length = NOALLOC_CHUNK;
    const size_t need = compressstore_workspace_size(n, elem_bytes, &cfg);
    if (need == 0) return CS_ERR_INVALID_VALUE;                 // bad elem_bytes
    if (need > NOALLOC_SCRATCH_BYTES) return CS_ERR_NOT_SUPPORTED; // unreachable for n <= NOALLOC_MAX_N
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return CS_ERR_NO_DEVICE;
    // the array's address on the current device, taken afresh on every call
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) {
        cudaGetLastError();
        return CS_ERR_CUDA;
    }
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        DeviceScratch& ds = g_noalloc_dev[dev];
        if (!ds.ready || ds.ptr != p) {
            // first call on this device, or the module was reloaded: zero the array, in
            // stream order ahead of this call's kernels
            const int st = cs_workspace_init(p, NOALLOC_SCRATCH_BYTES, stream);
            if (st != CS_SUCCESS) return st;
            ds.ptr = p;
            ds.ready = true;
        }
    }
    return compressstore_ex(d_in, d_mask, d_out, n, elem_bytes, d_count, p, NOALLOC_SCRATCH_BYTES, &cfg, stream);
}

} // extern "C"
