// cs_cub_flagged.cu — comparator only (not the product path): CUB DeviceSelect::Flagged
// over the same LSB-first packed uint32 mask, the bar the hand-written kernels are measured
// against. Reference: bitstream_iterator + launch_cub_flagged_biterator / bench8_cub_flagged
// (src/cub_wraps.cuh:12-50,81-99; src/benchmarks.cuh:384-394), which read an MSB-first
// byte mask; this iterator reads bit (i % 32) of word (i / 32).
#include <cstdint>
#include <iterator>

#include <cub/device/device_select.cuh>
#include <cuda_runtime.h>

#if defined(__GNUC__)
#define CSC_API extern "C" __attribute__((visibility("default")))
#else
#define CSC_API extern "C"
#endif

namespace {

struct LsbBitIterator {
    using value_type = bool;
    using reference = bool;
    using pointer = void;
    using difference_type = std::ptrdiff_t;
    using iterator_category = std::random_access_iterator_tag;

    const uint32_t* words;
    int64_t idx;

    __host__ __device__ LsbBitIterator(const uint32_t* w = nullptr, int64_t i = 0) : words(w), idx(i) {}
    __host__ __device__ bool operator[](int64_t i) const
    {
        const int64_t k = idx + i;
        return (words[k >> 5] >> (k & 31)) & 1u;
    }
    __host__ __device__ bool operator*() const { return (*this)[0]; }
    __host__ __device__ LsbBitIterator operator+(int64_t i) const { return LsbBitIterator(words, idx + i); }
    __host__ __device__ LsbBitIterator operator-(int64_t i) const { return LsbBitIterator(words, idx - i); }
    __host__ __device__ int64_t operator-(const LsbBitIterator& o) const { return idx - o.idx; }
    __host__ __device__ LsbBitIterator& operator++()
    {
        ++idx;
        return *this;
    }
    __host__ __device__ LsbBitIterator& operator+=(int64_t i)
    {
        idx += i;
        return *this;
    }
};

template <typename T>
cudaError_t run(void* d_temp, size_t& temp_bytes, const void* d_in, const uint32_t* d_mask, void* d_out,
                uint64_t* d_count, uint64_t n, cudaStream_t stream)
{
    return cub::DeviceSelect::Flagged(d_temp, temp_bytes, static_cast<const T*>(d_in), LsbBitIterator(d_mask, 0),
                                      static_cast<T*>(d_out), d_count, static_cast<int64_t>(n), stream);
}

cudaError_t dispatch(void* d_temp, size_t& temp_bytes, const void* d_in, const uint32_t* d_mask, void* d_out,
                     uint64_t* d_count, uint64_t n, uint32_t elem_bytes, cudaStream_t stream)
{
    switch (elem_bytes) {
        case 1: return run<uint8_t>(d_temp, temp_bytes, d_in, d_mask, d_out, d_count, n, stream);
        case 2: return run<uint16_t>(d_temp, temp_bytes, d_in, d_mask, d_out, d_count, n, stream);
        case 4: return run<uint32_t>(d_temp, temp_bytes, d_in, d_mask, d_out, d_count, n, stream);
        case 8: return run<uint64_t>(d_temp, temp_bytes, d_in, d_mask, d_out, d_count, n, stream);
        default: return cudaErrorInvalidValue;
    }
}

} // namespace

// Temporary storage bytes CUB needs for (n, elem_bytes); 0 on error.
CSC_API size_t cs_cub_flagged_temp_bytes(uint64_t n, uint32_t elem_bytes)
{
    size_t bytes = 0;
    if (dispatch(nullptr, bytes, nullptr, nullptr, nullptr, nullptr, n, elem_bytes, nullptr) != cudaSuccess) return 0;
    return bytes;
}

// Returns 0 on success, -4 on a CUDA error.
CSC_API int cs_cub_flagged(const void* d_in, const uint32_t* d_mask, void* d_out, uint64_t n, uint32_t elem_bytes,
                           uint64_t* d_count, void* d_temp, size_t temp_bytes, void* stream)
{
    size_t b = temp_bytes;
    const cudaError_t e =
        dispatch(d_temp, b, d_in, d_mask, d_out, d_count, n, elem_bytes, reinterpret_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? 0 : -4;
}
