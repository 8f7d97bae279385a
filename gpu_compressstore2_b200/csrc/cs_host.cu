// cs_host.cu — compaction of a HOST-resident column through the device.
//
// The column is streamed in pieces through SLOTS device buffers on three streams:
//   h2d     : payload + mask of piece i  (waits until slot i % SLOTS was drained)
//   compute : compaction of piece i into the slot's output, then its count to pinned host
//   d2h     : exactly count_i selected elements to h_out + (sum of earlier counts)
// The host thread waits only for each piece's count (to size and place its copy back), so
// host->device copies of later pieces, compaction, and device->host copies of earlier
// pieces overlap: with pinned host buffers the time approaches the larger of the two PCIe
// directions. The reference has no host-buffer path; its driver copies the whole column in
// and the validation out synchronously (src/main.cu:84-127, src/utils.cuh:41-48).
#include <cstring>
#include <map>
#include <mutex>

#include <cuda_runtime.h>

#include "compressstore.h"
#include "cs_internal.cuh"

namespace {

constexpr int SLOTS = 3;
constexpr uint64_t PIECE_BYTES = 32ull << 20; // payload bytes per piece

struct HostState {
    cudaStream_t h2d = nullptr, comp = nullptr, d2h = nullptr;
    cudaEvent_t loaded[SLOTS] = {};
    cudaEvent_t counted[SLOTS] = {};
    cudaEvent_t drained[SLOTS] = {};
    void* d_in[SLOTS] = {};
    void* d_mask[SLOTS] = {};
    void* d_out[SLOTS] = {};
    uint64_t* d_count = nullptr;  // SLOTS words
    uint64_t* h_count = nullptr;  // pinned, SLOTS words
    uint64_t piece_bytes = 0;
    std::mutex mu;
    bool ok = false;
};

std::mutex g_mu;
std::map<int, HostState*> g_states;

int status_of(cudaError_t e)
{
    if (e == cudaSuccess) return CS_SUCCESS;
    if (e == cudaErrorMemoryAllocation) return CS_ERR_OUT_OF_MEMORY;
    return CS_ERR_CUDA;
}

HostState* state_for(int dev, int* st)
{
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_states.find(dev);
    if (it != g_states.end()) {
        *st = it->second->ok ? CS_SUCCESS : CS_ERR_CUDA;
        return it->second;
    }
    auto s = new HostState();
    cudaError_t e = cudaSuccess;
    const unsigned fl = cudaStreamNonBlocking;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->h2d, fl);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->comp, fl);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->d2h, fl);
    s->piece_bytes = PIECE_BYTES;
    for (int i = 0; i < SLOTS && e == cudaSuccess; ++i) {
        e = cudaEventCreateWithFlags(&s->loaded[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->counted[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->drained[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&s->d_in[i], PIECE_BYTES);
        if (e == cudaSuccess) e = cudaMalloc(&s->d_mask[i], PIECE_BYTES / 8 + 256);
        if (e == cudaSuccess) e = cudaMalloc(&s->d_out[i], PIECE_BYTES);
    }
    if (e == cudaSuccess) e = cudaMalloc(&s->d_count, SLOTS * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_count, SLOTS * sizeof(uint64_t));
    s->ok = e == cudaSuccess;
    if (!s->ok) cudaGetLastError();
    g_states[dev] = s;
    *st = s->ok ? CS_SUCCESS : status_of(e);
    return s;
}

void destroy_state(HostState* s)
{
    if (s->h2d) cudaStreamSynchronize(s->h2d);
    if (s->comp) cudaStreamSynchronize(s->comp);
    if (s->d2h) cudaStreamSynchronize(s->d2h);
    if (s->comp) compressstore_release(reinterpret_cast<cs_stream_t>(s->comp));
    if (s->comp) cudaStreamSynchronize(s->comp);
    for (int i = 0; i < SLOTS; ++i) {
        if (s->loaded[i]) cudaEventDestroy(s->loaded[i]);
        if (s->counted[i]) cudaEventDestroy(s->counted[i]);
        if (s->drained[i]) cudaEventDestroy(s->drained[i]);
        if (s->d_in[i]) cudaFree(s->d_in[i]);
        if (s->d_mask[i]) cudaFree(s->d_mask[i]);
        if (s->d_out[i]) cudaFree(s->d_out[i]);
    }
    if (s->d_count) cudaFree(s->d_count);
    if (s->h_count) cudaFreeHost(s->h_count);
    if (s->h2d) cudaStreamDestroy(s->h2d);
    if (s->comp) cudaStreamDestroy(s->comp);
    if (s->d2h) cudaStreamDestroy(s->d2h);
    delete s;
}

} // namespace

extern "C" {

int compressstore_host_release(void)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CS_ERR_NO_DEVICE;
    HostState* s = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_states.find(dev);
        if (it == g_states.end()) return CS_SUCCESS;
        s = it->second;
        g_states.erase(it);
    }
    {
        std::lock_guard<std::mutex> lk(s->mu); // waits for a call in progress
    }
    destroy_state(s);
    return CS_SUCCESS;
}

int compressstore_host(const void* h_in, const void* h_mask, void* h_out, uint64_t n, uint32_t elem_bytes,
                       uint64_t* h_count, const cs_config* cfg)
{
    if (elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4 && elem_bytes != 8) return CS_ERR_INVALID_VALUE;
    if (!h_count) return CS_ERR_INVALID_VALUE;
    if (n == 0) {
        *h_count = 0;
        return CS_SUCCESS;
    }
    if (!h_in || !h_mask || !h_out) return CS_ERR_INVALID_VALUE;
    if ((reinterpret_cast<uintptr_t>(h_mask) & 3u) != 0) return CS_ERR_MISALIGNED;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return CS_ERR_NO_DEVICE;
    int st = CS_SUCCESS;
    HostState* s = state_for(dev, &st);
    if (st) return st;
    std::lock_guard<std::mutex> lk(s->mu);

    const uint64_t P = s->piece_bytes / elem_bytes; // elements per piece (a multiple of 4096)
    const uint64_t pieces = (n + P - 1) / P;
    const uint8_t* in = static_cast<const uint8_t*>(h_in);
    const uint8_t* mask = static_cast<const uint8_t*>(h_mask);
    uint8_t* out = static_cast<uint8_t*>(h_out);
    cudaError_t e = cudaSuccess;

    auto enqueue = [&](uint64_t i) -> int {
        const int k = static_cast<int>(i % SLOTS);
        const uint64_t e0 = i * P;
        const uint64_t ni = (n - e0) < P ? (n - e0) : P;
        // the slot's previous piece must have been copied out before it is overwritten
        if (i >= SLOTS) {
            e = cudaStreamWaitEvent(s->h2d, s->drained[k], 0);
            if (e != cudaSuccess) return status_of(e);
        }
        e = cudaMemcpyAsync(s->d_in[k], in + e0 * elem_bytes, ni * elem_bytes, cudaMemcpyHostToDevice, s->h2d);
        if (e != cudaSuccess) return status_of(e);
        e = cudaMemcpyAsync(s->d_mask[k], mask + e0 / 8, ((ni + 31) / 32) * 4, cudaMemcpyHostToDevice, s->h2d);
        if (e != cudaSuccess) return status_of(e);
        e = cudaEventRecord(s->loaded[k], s->h2d);
        if (e != cudaSuccess) return status_of(e);
        e = cudaStreamWaitEvent(s->comp, s->loaded[k], 0);
        if (e != cudaSuccess) return status_of(e);
        const int rc = compressstore_cfg(s->d_in[k], s->d_mask[k], s->d_out[k], ni, elem_bytes, s->d_count + k, cfg,
                                         reinterpret_cast<cs_stream_t>(s->comp));
        if (rc) return rc;
        e = cudaMemcpyAsync(s->h_count + k, s->d_count + k, sizeof(uint64_t), cudaMemcpyDeviceToHost, s->comp);
        if (e != cudaSuccess) return status_of(e);
        e = cudaEventRecord(s->counted[k], s->comp);
        return status_of(e);
    };

    // on failure, let everything already queued finish before the caller's buffers go away
    auto fail = [&](int rc) -> int {
        cudaStreamSynchronize(s->h2d);
        cudaStreamSynchronize(s->comp);
        cudaStreamSynchronize(s->d2h);
        return rc;
    };
    uint64_t total = 0;
    for (uint64_t i = 0; i < pieces && i < (uint64_t)SLOTS; ++i) {
        st = enqueue(i);
        if (st) return fail(st);
    }
    for (uint64_t j = 0; j < pieces; ++j) {
        const int k = static_cast<int>(j % SLOTS);
        e = cudaEventSynchronize(s->counted[k]);
        if (e != cudaSuccess) return fail(status_of(e));
        const uint64_t cj = s->h_count[k];
        if (cj == CS_COUNT_ERROR) {
            fail(0);
            const int rc = compressstore_check(reinterpret_cast<cs_stream_t>(s->comp));
            return rc ? rc : CS_ERR_TIMEOUT;
        }
        e = cudaStreamWaitEvent(s->d2h, s->counted[k], 0);
        if (e != cudaSuccess) return fail(status_of(e));
        if (cj) {
            e = cudaMemcpyAsync(out + total * elem_bytes, s->d_out[k], cj * elem_bytes, cudaMemcpyDeviceToHost, s->d2h);
            if (e != cudaSuccess) return fail(status_of(e));
        }
        e = cudaEventRecord(s->drained[k], s->d2h);
        if (e != cudaSuccess) return fail(status_of(e));
        total += cj;
        if (j + SLOTS < pieces) {
            st = enqueue(j + SLOTS);
            if (st) return fail(st);
        }
    }
    e = cudaStreamSynchronize(s->d2h);
    if (e != cudaSuccess) return status_of(e);
    st = compressstore_check(reinterpret_cast<cs_stream_t>(s->comp));
    if (st) return st;
    *h_count = total;
    return CS_SUCCESS;
}

} // extern "C"
