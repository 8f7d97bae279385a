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
// the last CTA of each kernel. It is zeroed once, when the first call on a device sets it
// up. Calls that overlap on the GPU (for example on two streams) race on that scratch and
// must not be made.
#include <mutex>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = 4u << 20; // 4 MiB per device
constexpr uint64_t NOALLOC_MAX_N = 1ull << 30;      // fits NOALLOC_SCRATCH_BYTES for every width
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
    const size_t need = compressstore_workspace_size(n, elem_bytes, nullptr);
    if (need == 0) return CS_ERR_INVALID_VALUE; // bad elem_bytes
    if (need > NOALLOC_SCRATCH_BYTES) return CS_ERR_NOT_SUPPORTED;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return CS_ERR_NO_DEVICE;
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        DeviceScratch& ds = g_noalloc_dev[dev];
        if (!ds.ready) {
            // first call on this device (it is current): find the array and zero it,
            // in stream order ahead of this call's kernels
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) {
                cudaGetLastError();
                return CS_ERR_CUDA;
            }
            const int st = cs_workspace_init(p, NOALLOC_SCRATCH_BYTES, stream);
            if (st != CS_SUCCESS) return st;
            ds.ptr = p;
            ds.ready = true;
        }
        scratch = ds.ptr;
    }
    return compressstore_ex(d_in, d_mask, d_out, n, elem_bytes, d_count, scratch, NOALLOC_SCRATCH_BYTES, nullptr,
                            stream);
}

} // extern "C"
