// ref_shim.cpp — TEST INFRASTRUCTURE ONLY. Exposes the reference's own CPU code for the
// compaction path (compiled from its sources where they lie, by oracle/Makefile) through
// a C ABI, so the oracle restatement can be checked against it and so the bench can time
// it as the CPU baseline. Nothing here is part of the product.
//
// Wrapped reference functions (RememberOfLife/gpu_compressstore2):
//   generate_validation<T>    src/data_generator.cuh:171-188  (sequential CPU compaction)
//   generate_mask_uniform     src/data_generator.cuh:14-31    (PCG32 mask, seed 42)
//   generate_mask_clustering  src/data_generator.cuh:130-167  (dense cluster masks)
//   generate_mask_pattern     src/data_generator.cuh:113-128  (periodic masks, pattern from the MSB)
// The reference reads masks MSB-first within each byte; callers pass such masks.
#define __host__
#define __device__
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "src/data_generator.cuh"

#define REF_API extern "C" __attribute__((visibility("default")))

namespace {
template <typename T>
uint64_t validation(const void* data, const uint8_t* mask_msb, void* out, uint64_t count)
{
    return generate_validation<T>(static_cast<T*>(const_cast<void*>(data)), const_cast<uint8_t*>(mask_msb),
                                  static_cast<T*>(out), count);
}

uint64_t validation_w(const void* data, const uint8_t* mask_msb, void* out, uint64_t count, uint32_t w)
{
    switch (w) {
        case 1: return validation<uint8_t>(data, mask_msb, out, count);
        case 2: return validation<uint16_t>(data, mask_msb, out, count);
        case 4: return validation<uint32_t>(data, mask_msb, out, count);
        case 8: return validation<uint64_t>(data, mask_msb, out, count);
        default: return 0;
    }
}
} // namespace

// generate_validation for element width w. `out` must hold `count` elements (the
// reference zero-fills everything past the selected ones). count should be a multiple of
// 8: the reference ignores a partial last mask byte.
REF_API uint64_t ref_generate_validation(const void* data, const uint8_t* mask_msb, void* out, uint64_t count,
                                         uint32_t elem_bytes)
{
    return validation_w(data, mask_msb, out, count, elem_bytes);
}

// The reference's CPU compaction run on `threads` host threads: every thread runs the
// reference's generate_validation on its own 8-element-aligned slice into a scratch
// buffer at the slice's start, then the slices are stitched to their output offsets.
// `scratch` must hold `count` elements.
REF_API uint64_t ref_generate_validation_mt(const void* data, const uint8_t* mask_msb, void* out, void* scratch,
                                            uint64_t count, uint32_t elem_bytes, int threads)
{
    if (threads < 1) threads = 1;
    const uint64_t bytes = count / 8;
    if (bytes == 0) return 0;
    if (static_cast<uint64_t>(threads) > bytes) threads = static_cast<int>(bytes);
    std::vector<uint64_t> b0(threads), cnt(threads), off(threads);
    for (int t = 0; t < threads; ++t) b0[t] = bytes * t / threads;
    auto slice_len = [&](int t) { return ((t + 1 < threads) ? b0[t + 1] : bytes) - b0[t]; };
    const uint8_t* d = static_cast<const uint8_t*>(data);
    uint8_t* s = static_cast<uint8_t*>(scratch);
    uint8_t* o = static_cast<uint8_t*>(out);
    std::vector<std::thread> th;
    for (int t = 0; t < threads; ++t)
        th.emplace_back([&, t] {
            const uint64_t e0 = b0[t] * 8;
            cnt[t] = validation_w(d + e0 * elem_bytes, mask_msb + b0[t], s + e0 * elem_bytes, slice_len(t) * 8,
                                  elem_bytes);
        });
    for (auto& x : th) x.join();
    th.clear();
    uint64_t run = 0;
    for (int t = 0; t < threads; ++t) {
        off[t] = run;
        run += cnt[t];
    }
    for (int t = 0; t < threads; ++t)
        th.emplace_back([&, t] {
            std::memcpy(o + off[t] * elem_bytes, s + b0[t] * 8 * elem_bytes, cnt[t] * elem_bytes);
        });
    for (auto& x : th) x.join();
    return run;
}

REF_API uint64_t ref_generate_mask_uniform(uint8_t* buf, uint64_t offset, uint64_t length, double selectivity)
{
    size_t ones = 0;
    generate_mask_uniform(buf, offset, length, selectivity, &ones);
    return ones;
}

// generate_mask_clustering(selectivity, cluster_count, total_elements); writes
// total_elements/8 bytes to out and returns the number of ones.
REF_API uint64_t ref_generate_mask_clustering(float selectivity, uint64_t cluster_count, uint64_t total_elements,
                                              uint8_t* out)
{
    size_t ones = 0;
    std::vector<uint8_t> m = generate_mask_clustering(selectivity, cluster_count, total_elements, &ones);
    std::memcpy(out, m.data(), m.size());
    return ones;
}

// The reference's periodic mask: `bytes` MSB-first mask bytes, element i selected when bit
// 31 - (i % length) of `pattern` is set. Returns the number of selected elements.
REF_API uint64_t ref_generate_mask_pattern(uint8_t* out, uint64_t bytes, uint32_t pattern, uint32_t length)
{
    size_t ones = 0;
    generate_mask_pattern(out, 0, bytes, pattern, length, &ones);
    return ones;
}
