// cs_tuning.cu — the CS_ALGO_AUTO table and its run-time override entry points.
#include <atomic>
#include <cstdint>

#include "compressstore.h"
#include "cs_tuning.h"

namespace cs {

namespace {
// Packed entry: algo in bits 0..7, log2(chunk_length) in bits 8..15. Zero = unset.
std::atomic<uint32_t> g_table[TUNE_WIDTHS][TUNE_SIZES];

TuneChoice default_choice(uint64_t n, uint32_t elem_bytes)
{
    (void)n;
    (void)elem_bytes;
    return TuneChoice{CS_ALGO_3PASS, 1024u};
}
} // namespace

int tune_width_index(uint32_t elem_bytes)
{
    switch (elem_bytes) {
        case 1: return 0;
        case 2: return 1;
        case 4: return 2;
        case 8: return 3;
        default: return -1;
    }
}

int tune_size_bucket(uint64_t n)
{
    int lg = 0;
    while (lg < 63 && (1ull << (lg + 1)) <= n) ++lg;
    int b = lg / 2;
    if (b >= TUNE_SIZES) b = TUNE_SIZES - 1;
    return b;
}

TuneChoice tune_lookup(uint64_t n, uint32_t elem_bytes)
{
    const int wi = tune_width_index(elem_bytes);
    if (wi < 0) return default_choice(n, elem_bytes);
    const uint32_t e = g_table[wi][tune_size_bucket(n)].load(std::memory_order_relaxed);
    if (e == 0) return default_choice(n, elem_bytes);
    return TuneChoice{static_cast<int>(e & 0xffu), 1u << ((e >> 8) & 0xffu)};
}

} // namespace cs

extern "C" {

int cs_tune_set(uint32_t elem_bytes, int32_t size_bucket, int32_t algo, uint32_t chunk_length)
{
    const int wi = cs::tune_width_index(elem_bytes);
    if (wi < 0 || size_bucket < 0 || size_bucket >= cs::TUNE_SIZES) return CS_ERR_INVALID_VALUE;
    if (algo == CS_ALGO_AUTO) {
        cs::g_table[wi][size_bucket].store(0u);
        return CS_SUCCESS;
    }
    if (algo < CS_ALGO_1PASS || algo > CS_ALGO_NAIVE) return CS_ERR_INVALID_VALUE;
    if (chunk_length < 32 || chunk_length > 65536 || (chunk_length & (chunk_length - 1))) return CS_ERR_INVALID_VALUE;
    uint32_t lg = 0;
    while ((1u << lg) < chunk_length) ++lg;
    cs::g_table[wi][size_bucket].store(static_cast<uint32_t>(algo) | (lg << 8));
    return CS_SUCCESS;
}

int cs_tune_get(uint32_t elem_bytes, uint64_t n, int32_t* algo, uint32_t* chunk_length)
{
    if (cs::tune_width_index(elem_bytes) < 0 || !algo || !chunk_length) return CS_ERR_INVALID_VALUE;
    const cs::TuneChoice t = cs::tune_lookup(n, elem_bytes);
    *algo = t.algo;
    *chunk_length = t.chunk_length;
    return CS_SUCCESS;
}

int cs_tune_size_bucket(uint64_t n)
{
    return cs::tune_size_bucket(n);
}

} // extern "C"
