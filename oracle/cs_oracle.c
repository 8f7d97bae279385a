/*
 * cs_oracle.c — CPU oracle for bitmask stream compaction. TEST INFRASTRUCTURE ONLY:
 * it is the checker the GPU kernels are compared against (tests, smoke check, and the
 * bench's CPU baseline leg). The product never calls it.
 *
 * Parity is pinned two ways (tests/test_oracle.py):
 *   - against the reference's own CPU code compiled here from its sources
 *     (oracle/_ref/libcsref.so, built by oracle/Makefile from ref_shim.cpp), run on the
 *     per-byte bit-reversed mask because the reference packs bits MSB-first;
 *   - against committed golden vectors in tests/golden/ generated from that build by
 *     tests/golden/make_golden.py, and the reference-derived known answers
 *     (uniform seed-42 mask bytes 09 f7 bb 9f 36 fc b4 34; mask {0x81,0x40} over
 *     100+i selects {100,107,109}).
 *
 * Mask convention here: uint32 words, LSB-first; bit (i % 32) of word (i / 32) selects
 * element i. Bits at positions >= n are ignored.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------------------------
 * Compaction. Restates generate_validation<T> (src/data_generator.cuh:171-188): walk the
 * mask in element order, append every selected element, return the number selected.
 * Differences, all deliberate: LSB-first uint32 words instead of MSB-first bytes; the
 * partial last byte/word is honoured (the reference loops count/8 full bytes only,
 * :175); the count is 64-bit (the reference accumulates a uint32_t, :173); nothing is
 * written past the count (the reference zero-fills the rest of its buffer, :186).
 * ---------------------------------------------------------------------------------- */
static inline uint32_t word_at(const uint32_t* mask, uint64_t wi, uint64_t n)
{
    uint64_t nw = (n + 31) / 32;
    uint32_t m = mask[wi];
    if (wi == nw - 1 && (n & 31u)) m &= (1u << (n & 31u)) - 1u;
    return m;
}

static uint64_t compact_range(const uint8_t* in, const uint32_t* mask, uint8_t* out, uint64_t n, uint32_t w,
                              uint64_t w_begin, uint64_t w_end)
{
    uint64_t k = 0;
    for (uint64_t wi = w_begin; wi < w_end; ++wi) {
        uint32_t m = word_at(mask, wi, n);
        while (m) {
            const uint32_t b = (uint32_t)__builtin_ctz(m);
            const uint64_t i = wi * 32 + b;
            switch (w) {
                case 1: out[k] = in[i]; break;
                case 2: memcpy(out + 2 * k, in + 2 * i, 2); break;
                case 4: memcpy(out + 4 * k, in + 4 * i, 4); break;
                default: memcpy(out + 8 * k, in + 8 * i, 8); break;
            }
            ++k;
            m &= m - 1;
        }
    }
    return k;
}

ORACLE_API uint64_t oracle_compact(const void* in, const uint32_t* mask, void* out, uint64_t n, uint32_t elem_bytes)
{
    if (n == 0) return 0;
    return compact_range((const uint8_t*)in, mask, (uint8_t*)out, n, elem_bytes, 0, (n + 31) / 32);
}

ORACLE_API uint64_t oracle_count(const uint32_t* mask, uint64_t n)
{
    uint64_t c = 0;
    const uint64_t nw = (n + 31) / 32;
    for (uint64_t wi = 0; wi < nw; ++wi) c += (uint64_t)__builtin_popcount(word_at(mask, wi, n));
    return c;
}

/* Multi-threaded restatement for the timed CPU baseline: count per slice -> exclusive
 * prefix -> each thread copies its slice to its offset. */
typedef struct {
    const uint8_t* in;
    const uint32_t* mask;
    uint8_t* out;
    uint64_t n;
    uint32_t w;
    uint64_t w_begin, w_end;
    uint64_t count;
    uint64_t offset;
    int phase;
} slice_t;

static void* slice_run(void* arg)
{
    slice_t* s = (slice_t*)arg;
    if (s->phase == 0) {
        uint64_t c = 0;
        for (uint64_t wi = s->w_begin; wi < s->w_end; ++wi) c += (uint64_t)__builtin_popcount(word_at(s->mask, wi, s->n));
        s->count = c;
    } else {
        compact_range(s->in, s->mask, s->out + s->offset * s->w, s->n, s->w, s->w_begin, s->w_end);
    }
    return NULL;
}

ORACLE_API uint64_t oracle_compact_mt(const void* in, const uint32_t* mask, void* out, uint64_t n, uint32_t elem_bytes,
                                      int threads)
{
    if (n == 0) return 0;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    const uint64_t nw = (n + 31) / 32;
    if ((uint64_t)threads > nw) threads = (int)nw;
    slice_t sl[256];
    pthread_t th[256];
    for (int t = 0; t < threads; ++t) {
        sl[t].in = (const uint8_t*)in;
        sl[t].mask = mask;
        sl[t].out = (uint8_t*)out;
        sl[t].n = n;
        sl[t].w = elem_bytes;
        sl[t].w_begin = nw * (uint64_t)t / (uint64_t)threads;
        sl[t].w_end = nw * (uint64_t)(t + 1) / (uint64_t)threads;
        sl[t].phase = 0;
    }
    for (int phase = 0; phase < 2; ++phase) {
        if (phase == 1) {
            uint64_t off = 0;
            for (int t = 0; t < threads; ++t) {
                sl[t].offset = off;
                off += sl[t].count;
            }
        }
        for (int t = 0; t < threads; ++t) {
            sl[t].phase = phase;
            pthread_create(&th[t], NULL, slice_run, &sl[t]);
        }
        for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
    }
    uint64_t total = 0;
    for (int t = 0; t < threads; ++t) total += sl[t].count;
    return total;
}

/* Pass 1 restated: kernel_3pass_popc_none_striding (src/kernels/kernel_3pass.cuh:12-38),
 * count per chunk of chunk_length elements. */
ORACLE_API void oracle_popc_chunks(const uint32_t* mask, uint64_t n, uint32_t chunk_length, uint32_t* counts)
{
    const uint64_t chunks = (n + chunk_length - 1) / chunk_length;
    const uint64_t wpc = chunk_length / 32;
    const uint64_t nw = (n + 31) / 32;
    for (uint64_t c = 0; c < chunks; ++c) {
        uint32_t s = 0;
        for (uint64_t wi = c * wpc; wi < (c + 1) * wpc && wi < nw; ++wi) s += (uint32_t)__builtin_popcount(word_at(mask, wi, n));
        counts[c] = s;
    }
}

/* Pass 2 restated: exclusive prefix sum of the chunk counts (the reference uses
 * cub::DeviceScan::ExclusiveSum, src/cub_wraps.cuh:61-68, or its up-sweep tree,
 * src/kernels/kernel_3pass.cuh:69-214). */
ORACLE_API uint64_t oracle_exclusive_scan(const uint32_t* counts, uint64_t c, uint64_t* offsets)
{
    uint64_t run = 0;
    for (uint64_t i = 0; i < c; ++i) {
        offsets[i] = run;
        run += counts[i];
    }
    return run;
}

/* ------------------------------------------------------------------------------------
 * Seeded generators (the same counter-based definitions the device generators use).
 * mix64 is the SplitMix64 output function (Steele, Lea, Flood 2014) on
 * seed + (i+1)*0x9E3779B97F4A7C15.
 * ---------------------------------------------------------------------------------- */
ORACLE_API uint64_t oracle_mix64(uint64_t seed, uint64_t i)
{
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

ORACLE_API void oracle_gen_payload(void* out, uint64_t n, uint32_t elem_bytes, uint64_t seed, int float_unit)
{
    uint8_t* o = (uint8_t*)out;
    for (uint64_t i = 0; i < n; ++i) {
        const uint64_t h = oracle_mix64(seed, i);
        if (elem_bytes == 4 && float_unit) {
            float f = (float)(uint32_t)(h >> 40) * (1.0f / 16777216.0f);
            memcpy(o + 4 * i, &f, 4);
        } else {
            memcpy(o + (uint64_t)elem_bytes * i, &h, elem_bytes); /* little-endian low bytes */
        }
    }
}

static uint64_t bernoulli_threshold(double p)
{
    if (p >= 1.0) return 1ull << 32;
    if (p <= 0.0) return 0;
    return (uint64_t)(p * 4294967296.0);
}

ORACLE_API void oracle_gen_mask_bernoulli(uint32_t* mask, uint64_t n, double p, uint64_t seed)
{
    const uint64_t thr = bernoulli_threshold(p);
    const uint64_t nw = (n + 31) / 32;
    for (uint64_t w = 0; w < nw; ++w) {
        uint32_t m = 0;
        for (uint32_t b = 0; b < 32; ++b) {
            const uint64_t i = w * 32 + b;
            if (i < n && (oracle_mix64(seed, i) >> 32) < thr) m |= 1u << b;
        }
        mask[w] = m;
    }
}

/* Alternating runs: position i toggles the state with probability 1/mean_run; bit i is
 * the state after position i (the xor of all toggles up to and including i). */
ORACLE_API void oracle_gen_mask_runs(uint32_t* mask, uint64_t n, double mean_run, uint64_t seed)
{
    const uint64_t thr = (uint64_t)(4294967296.0 / mean_run);
    const uint64_t nw = (n + 31) / 32;
    uint32_t state = 0;
    for (uint64_t w = 0; w < nw; ++w) {
        uint32_t m = 0;
        for (uint32_t b = 0; b < 32; ++b) {
            const uint64_t i = w * 32 + b;
            if (i >= n) break;
            if ((oracle_mix64(seed, i) >> 32) < thr) state ^= 1u;
            m |= state << b;
        }
        mask[w] = m;
    }
}

/* Single dense block at the front: k = (size_t)((float)frac * (float)n) leading ones,
 * the rounding of generate_mask_clustering(frac, 1, n) (src/data_generator.cuh:130-167,
 * total_set_one = selectivity * total_elements in float). */
ORACLE_API uint64_t oracle_gen_mask_dense_prefix(uint32_t* mask, uint64_t n, float frac)
{
    uint64_t k = (uint64_t)(frac * (float)n);
    if (k > n) k = n;
    const uint64_t nw = (n + 31) / 32;
    for (uint64_t w = 0; w < nw; ++w) {
        const uint64_t lo = w * 32;
        if (lo + 32 <= k) mask[w] = 0xffffffffu;
        else if (lo >= k) mask[w] = 0;
        else mask[w] = (1u << (k - lo)) - 1u;
    }
    return k;
}

/* Periodic mask, LSB-first words: bit i is bit (i % L) of `pattern` (1 <= L <= 32). The
 * reference builds the same selection MSB-first in bytes, element i <-> bit 31 - i % L of its
 * pattern (generate_mask_pattern, src/data_generator.cuh:113-128); the two agree when this
 * pattern is the bit reversal of the reference's. Returns the number of set bits. */
ORACLE_API uint64_t oracle_gen_mask_pattern(uint32_t* mask, uint64_t n, uint32_t pattern, uint32_t L)
{
    uint64_t ones = 0;
    const uint64_t nw = (n + 31) / 32;
    for (uint64_t w = 0; w < nw; ++w) {
        uint32_t m = 0;
        for (uint32_t b = 0; b < 32; ++b) {
            const uint64_t i = w * 32 + b;
            if (i < n && ((pattern >> (uint32_t)(i % L)) & 1u)) {
                m |= 1u << b;
                ++ones;
            }
        }
        mask[w] = m;
    }
    return ones;
}

/* ------------------------------------------------------------------------------------
 * The reference's PRNG, restated to pin known answers: PCG32 (XSH-RR, O'Neill 2014)
 * seeded through SplitMix64 as in src/fast_prng.cuh:7-36, and the MSB-first uniform
 * mask generator of src/data_generator.cuh:14-31.
 * ---------------------------------------------------------------------------------- */
typedef struct {
    uint64_t state, inc;
} pcg_t;

static void pcg_seed(pcg_t* r, uint64_t seed)
{
    uint64_t z = seed + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    r->state = z ^ (z >> 31);
    r->inc = 1;
}

static uint32_t pcg_next(pcg_t* r)
{
    const uint64_t old = r->state;
    r->state = old * 6364136223846793005ull + (r->inc | 1u);
    const uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31u));
}

ORACLE_API uint64_t oracle_ref_mask_uniform_msb(uint8_t* buf, uint64_t length, double selectivity, uint64_t seed)
{
    const uint64_t thr = (uint64_t)(selectivity * 4294967295.0);
    pcg_t r;
    pcg_seed(&r, seed);
    uint64_t ones = 0;
    for (uint64_t i = 0; i < length; ++i) {
        uint8_t acc = 0;
        for (int j = 7; j >= 0; --j) {
            if (pcg_next(&r) < thr) {
                acc |= (uint8_t)(1u << j);
                ++ones;
            }
        }
        buf[i] = acc;
    }
    return ones;
}

/* Adapter between the two packings: reverse the bit order inside every byte. An
 * LSB-first mask (bytes of the uint32 words, little-endian) becomes the reference's
 * MSB-first byte mask selecting the same elements, and back. */
ORACLE_API void oracle_rev8(uint8_t* bytes, uint64_t len)
{
    for (uint64_t i = 0; i < len; ++i) {
        uint8_t b = bytes[i];
        b = (uint8_t)(((b & 0xF0u) >> 4) | ((b & 0x0Fu) << 4));
        b = (uint8_t)(((b & 0xCCu) >> 2) | ((b & 0x33u) << 2));
        b = (uint8_t)(((b & 0xAAu) >> 1) | ((b & 0x55u) << 1));
        bytes[i] = b;
    }
}
