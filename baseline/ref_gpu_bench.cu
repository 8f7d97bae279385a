// ref_gpu_bench.cu — times the reference's OWN GPU compositions on this GPU. NOT PRODUCT:
// a comparator, built by baseline/Makefile from the reference's sources where they lie
// (nothing of them is copied here) and run by bench.py in a child process.
//
// Timed compositions (RememberOfLife/gpu_compressstore2, called unmodified through their
// own operator API, benchN(intermediate_data*, ...)):
//   bench10  src/benchmarks.cuh:418-440  popc -> CUB ExclusiveSum -> smem-staged writeout
//            (kernel_3pass_proc_true_striding_optimized_writeout, src/kernels/kernel_3pass.cuh:329-467)
//   bench7   src/benchmarks.cuh:360-382  popc -> CUB ExclusiveSum -> naive writeout
//            (src/kernels/kernel_3pass.cuh:216-327)
//   bench8   src/benchmarks.cuh:384-394  cub::DeviceSelect::Flagged over the reference's
//            bitstream_iterator (src/cub_wraps.cuh:12-50)
// The reference's scratch owner intermediate_data (src/benchmarks.cuh:53-151) is built as its
// driver builds it (src/main.cu:134: chunk_length_min 32, 8 streams).
//
// Inputs: the same seeded payload and LSB-first mask words as the library's bench
// (cs_gen_payload / cs_gen_mask_bernoulli of libcompressstore.so), the mask converted to the
// reference's MSB-first bytes (bit order reversed inside every byte). Every timed
// configuration's output is compared byte for byte with the library's plain call on the same
// inputs (whose own parity with the reference CPU code the GPU tests establish). The
// reference's count is not compared: its pssskip kernel double-adds the last chunk
// (src/benchmarks.cuh:430-433).
//
// The reference works in uint32 element indices and counts, so n must stay below 2^32; its
// kernels are instantiated here for 4-byte elements (float32 bits move as uint32) and 8-byte
// elements, as its driver does (src/main.cu:305-310). n must be a multiple of 8192 so every
// chunk length of the sweep (32 .. 8192) divides it; with that, every access the kernels make
// stays inside the buffers allocated here (popc reads n/8 mask bytes and writes n/L counts;
// the writeouts read input[< n] and write output[< count]).
//
// Output: one JSON object on stdout:
//   {"n", "elem_bytes", "p", "count", "results": [{"bench", "chunk", "block", "grid",
//    "total_ms_min", "total_ms_mean", "popc_ms", "proc_ms", "ok"}], "best": {bench: result}}
// total_ms is the reference's own timings.total (CUDA events around the whole composition,
// including its host-side synchronisations), the number its eval database records.
#include <algorithm>
#include <bitset> // the reference's headers use these without including them (its main.cu does first)
#include <cassert>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "src/benchmarks.cuh"

#include "compressstore.h"

namespace {

__global__ void k_rev8(const uint32_t* words, uint32_t* msb, uint64_t nwords)
{
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < nwords;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        // reverse all 32 bits, then the byte order back: each byte's bits end up reversed in place
        msb[i] = __byte_perm(__brev(words[i]), 0u, 0x0123u);
    }
}

__global__ void k_mismatch(const uint8_t* a, const uint8_t* b, uint64_t bytes, unsigned long long* bad)
{
    unsigned long long local = 0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < bytes;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        local += a[i] != b[i];
    if (local) atomicAdd(bad, local);
}

#define CHECK(x)                                                                                                       \
    do {                                                                                                               \
        cudaError_t e_ = (x);                                                                                          \
        if (e_ != cudaSuccess) {                                                                                       \
            fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_));                         \
            exit(3);                                                                                                   \
        }                                                                                                              \
    } while (0)

struct Result {
    std::string bench;
    int chunk, block, grid;
    double total_min, total_mean, popc, proc;
    bool ok;
};

std::vector<int> parse_list(const char* s)
{
    std::vector<int> v;
    const char* p = s;
    while (*p) {
        v.push_back(atoi(p));
        const char* c = strchr(p, ',');
        if (!c) break;
        p = c + 1;
    }
    return v;
}

template <typename T>
int run(uint64_t n, double p, uint64_t pseed, uint64_t mseed, int reps, const std::vector<int>& chunks,
        const std::vector<int>& blocks, const std::vector<int>& grids, const std::string& benches, const char* dump)
{
    const uint32_t w = sizeof(T);
    T *d_in = nullptr, *d_out = nullptr, *d_lib = nullptr;
    uint32_t *d_words = nullptr, *d_msb = nullptr;
    uint64_t* d_count = nullptr;
    unsigned long long* d_bad = nullptr;
    const uint64_t nwords = n / 32;
    CHECK(cudaMalloc(&d_in, n * w));
    CHECK(cudaMalloc(&d_out, n * w));
    CHECK(cudaMalloc(&d_lib, n * w));
    CHECK(cudaMalloc(&d_words, nwords * 4));
    CHECK(cudaMalloc(&d_msb, nwords * 4));
    CHECK(cudaMalloc(&d_count, 8));
    CHECK(cudaMalloc(&d_bad, 8));
    if (cs_gen_payload(d_in, n, w, pseed, w == 4 ? 1 : 0, nullptr) != CS_SUCCESS) return 4;
    if (cs_gen_mask_bernoulli(d_words, n, p, mseed, nullptr) != CS_SUCCESS) return 4;
    k_rev8<<<1184, 256>>>(d_words, d_msb, nwords);
    CHECK(cudaGetLastError());
    if (compressstore(d_in, d_words, d_lib, n, w, d_count, nullptr) != CS_SUCCESS) return 4;
    CHECK(cudaDeviceSynchronize());
    if (compressstore_check(nullptr) != CS_SUCCESS) return 4;
    uint64_t count = 0;
    CHECK(cudaMemcpy(&count, d_count, 8, cudaMemcpyDeviceToHost));

    intermediate_data id{n, 32, 8, static_cast<T*>(nullptr)};
    uint8_t* mask = reinterpret_cast<uint8_t*>(d_msb);
    std::vector<Result> results;
    auto verify = [&]() -> bool {
        CHECK(cudaMemset(d_bad, 0, 8));
        k_mismatch<<<1184, 256>>>(reinterpret_cast<const uint8_t*>(d_out), reinterpret_cast<const uint8_t*>(d_lib),
                                  count * w, d_bad);
        unsigned long long bad = 0;
        CHECK(cudaMemcpy(&bad, d_bad, 8, cudaMemcpyDeviceToHost));
        return bad == 0;
    };
    auto time_one = [&](const char* name, int L, int B, int G, auto&& fn) {
        timings warm = fn(L, B, G); // first call pays module loading and CUB set-up
        (void)warm;
        double tmin = 1e30, tsum = 0, popc = 0, proc = 0;
        for (int r = 0; r < reps; ++r) {
            const timings t = fn(L, B, G);
            tsum += t.total;
            if (t.total < tmin) {
                tmin = t.total;
                popc = t.popc;
                proc = t.proc;
            }
        }
        const bool ok = verify();
        results.push_back({name, L, B, G, tmin, tsum / reps, popc, proc, ok});
        if (dump) { // the composition's output of its last run, for a check against the CPU oracle
            std::vector<uint8_t> h(count * w);
            CHECK(cudaMemcpy(h.data(), d_out, h.size(), cudaMemcpyDeviceToHost));
            const std::string path = std::string(dump) + "_" + name + ".bin";
            FILE* f = fopen(path.c_str(), "wb");
            if (!f || fwrite(h.data(), 1, h.size(), f) != h.size()) {
                fprintf(stderr, "cannot write %s\n", path.c_str());
                exit(3);
            }
            fclose(f);
        }
    };
    auto want = [&](const char* b) { return benches.find(b) != std::string::npos; };
    if (want("bench8"))
        time_one("bench8", 0, 0, 0, [&](int, int, int) { return bench8_cub_flagged<T>(&id, d_in, mask, d_out, n); });
    for (int L : chunks)
        for (int B : blocks)
            for (int G : grids) {
                if (want("bench10"))
                    time_one("bench10", L, B, G, [&](int l, int b, int g) {
                        return bench10_3pass_optimized_read_skipping_optimized_writeout_cub_pss<T>(&id, d_in, mask,
                                                                                                  d_out, n, l, b, g);
                    });
                if (want("bench7"))
                    time_one("bench7", L, B, G, [&](int l, int b, int g) {
                        return bench7_3pass_optimized_read_skipping_cub_pss<T>(&id, d_in, mask, d_out, n, l, b, g);
                    });
            }
    CHECK(cudaDeviceSynchronize());

    printf("{\"n\": %llu, \"elem_bytes\": %u, \"p\": %g, \"count\": %llu, \"reps\": %d, \"results\": [",
           (unsigned long long)n, w, p, (unsigned long long)count, reps);
    for (size_t i = 0; i < results.size(); ++i) {
        const Result& r = results[i];
        printf("%s{\"bench\": \"%s\", \"chunk\": %d, \"block\": %d, \"grid\": %d, \"total_ms_min\": %.6f, "
               "\"total_ms_mean\": %.6f, \"popc_ms\": %.6f, \"proc_ms\": %.6f, \"ok\": %s}",
               i ? ", " : "", r.bench.c_str(), r.chunk, r.block, r.grid, r.total_min, r.total_mean, r.popc, r.proc,
               r.ok ? "true" : "false");
    }
    printf("], \"best\": {");
    bool first = true;
    for (const char* b : {"bench10", "bench7", "bench8"}) {
        const Result* best = nullptr;
        for (const Result& r : results)
            if (r.bench == b && r.ok && (!best || r.total_min < best->total_min)) best = &r;
        if (!best) continue;
        printf("%s\"%s\": {\"chunk\": %d, \"block\": %d, \"grid\": %d, \"total_ms_min\": %.6f, \"proc_ms\": %.6f}",
               first ? "" : ", ", b, best->chunk, best->block, best->grid, best->total_min, best->proc);
        first = false;
    }
    printf("}}\n");
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFree(d_lib);
    cudaFree(d_words);
    cudaFree(d_msb);
    cudaFree(d_count);
    cudaFree(d_bad);
    return 0;
}

} // namespace

// usage: ref_gpu_bench n elem_bytes p payload_seed mask_seed reps chunks blocks grids benches [dump]
//        (lists comma-separated; benches e.g. "bench10,bench7,bench8"; with dump, each bench's
//        output of its last timed run is written to <dump>_<bench>.bin)
int main(int argc, char** argv)
{
    if (argc < 11) {
        fprintf(stderr, "usage: %s n elem_bytes p payload_seed mask_seed reps chunks blocks grids benches\n", argv[0]);
        return 2;
    }
    const uint64_t n = strtoull(argv[1], nullptr, 10);
    const int w = atoi(argv[2]);
    const double p = atof(argv[3]);
    const uint64_t pseed = strtoull(argv[4], nullptr, 10), mseed = strtoull(argv[5], nullptr, 10);
    const int reps = std::max(1, atoi(argv[6]));
    const std::vector<int> chunks = parse_list(argv[7]), blocks = parse_list(argv[8]), grids = parse_list(argv[9]);
    const std::string benches = argv[10];
    const char* dump = argc > 11 ? argv[11] : nullptr;
    if (n == 0 || n % 8192 != 0 || n >= (1ull << 32)) {
        fprintf(stderr, "n must be a positive multiple of 8192 below 2^32 (the reference indexes in uint32)\n");
        return 2;
    }
    for (int L : chunks)
        if (L < 32 || L > 8192 || (L & (L - 1))) {
            fprintf(stderr, "chunk lengths: powers of two in [32, 8192] (the reference driver's sweep)\n");
            return 2;
        }
    for (int B : blocks)
        if (B < 32 || B > 1024 || (B & (B - 1))) {
            fprintf(stderr, "block sizes: powers of two in [32, 1024]\n");
            return 2;
        }
    for (int G : grids)
        if (G < 32 || G > 2048 || (G & (G - 1))) {
            fprintf(stderr, "grid sizes: powers of two in [32, 2048] (the reference driver's sweep)\n");
            return 2;
        }
    if (w == 4) return run<uint32_t>(n, p, pseed, mseed, reps, chunks, blocks, grids, benches, dump);
    if (w == 8) return run<uint64_t>(n, p, pseed, mseed, reps, chunks, blocks, grids, benches, dump);
    fprintf(stderr, "elem_bytes must be 4 or 8\n");
    return 2;
}
