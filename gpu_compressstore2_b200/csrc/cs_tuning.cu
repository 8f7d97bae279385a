// cs_tuning.cu — the CS_ALGO_AUTO table and its run-time override entry points.
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <mutex>

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

int load_table_file(const char* path);

// A table named by the CS_TUNE_TABLE environment variable is installed before the first
// lookup (entries set later with cs_tune_set / cs_tune_load override it).
void load_env_table_once()
{
    static std::once_flag once;
    std::call_once(once, [] {
        const char* p = std::getenv("CS_TUNE_TABLE");
        if (p && *p) load_table_file(p);
    });
}

int set_entry(uint32_t elem_bytes, int32_t size_bucket, int32_t algo, uint32_t chunk_length)
{
    const int wi = tune_width_index(elem_bytes);
    if (wi < 0 || size_bucket < 0 || size_bucket >= TUNE_SIZES) return CS_ERR_INVALID_VALUE;
    if (algo == CS_ALGO_AUTO) {
        g_table[wi][size_bucket].store(0u);
        return CS_SUCCESS;
    }
    if (algo < CS_ALGO_1PASS || algo > CS_ALGO_NAIVE) return CS_ERR_INVALID_VALUE;
    if (chunk_length < 32 || chunk_length > 65536 || (chunk_length & (chunk_length - 1))) return CS_ERR_INVALID_VALUE;
    uint32_t lg = 0;
    while ((1u << lg) < chunk_length) ++lg;
    g_table[wi][size_bucket].store(static_cast<uint32_t>(algo) | (lg << 8));
    return CS_SUCCESS;
}

// Text table: one entry per line, "elem_bytes size_bucket algo chunk_length"; '#' starts a
// comment. Every line is validated before any entry is installed.
int load_table_file(const char* path)
{
    FILE* f = std::fopen(path, "r");
    if (!f) return CS_ERR_INVALID_VALUE;
    struct Entry {
        uint32_t w;
        int32_t b, a;
        uint32_t c;
    };
    Entry entries[TUNE_WIDTHS * TUNE_SIZES];
    int count = 0, rc = CS_SUCCESS;
    char line[256];
    while (std::fgets(line, sizeof(line), f)) {
        char* hash = line;
        while (*hash && *hash != '#') ++hash;
        *hash = 0;
        unsigned w = 0, c = 0;
        int b = 0, a = 0;
        char extra = 0;
        const int got = std::sscanf(line, " %u %d %d %u %c", &w, &b, &a, &c, &extra);
        if (got <= 0) continue; // blank or comment line
        if (got != 4 || count == TUNE_WIDTHS * TUNE_SIZES || tune_width_index(w) < 0 || b < 0 || b >= TUNE_SIZES ||
            a < CS_ALGO_AUTO || a > CS_ALGO_NAIVE ||
            (a != CS_ALGO_AUTO && (c < 32 || c > 65536 || (c & (c - 1))))) {
            rc = CS_ERR_INVALID_VALUE;
            break;
        }
        entries[count++] = Entry{w, b, a, c};
    }
    std::fclose(f);
    if (rc != CS_SUCCESS) return rc;
    for (int i = 0; i < count; ++i) set_entry(entries[i].w, entries[i].b, entries[i].a, entries[i].c);
    return CS_SUCCESS;
}

TuneChoice tune_lookup(uint64_t n, uint32_t elem_bytes)
{
    load_env_table_once();
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
    cs::load_env_table_once(); // so that the environment's table cannot override this later
    return cs::set_entry(elem_bytes, size_bucket, algo, chunk_length);
}

int cs_tune_load(const char* path)
{
    if (!path) return CS_ERR_INVALID_VALUE;
    cs::load_env_table_once();
    return cs::load_table_file(path);
}

int cs_tune_save(const char* path)
{
    if (!path) return CS_ERR_INVALID_VALUE;
    cs::load_env_table_once();
    FILE* f = std::fopen(path, "w");
    if (!f) return CS_ERR_INVALID_VALUE;
    std::fprintf(f, "# elem_bytes size_bucket algo chunk_length  (size_bucket = floor(log2(n)) / 2)\n");
    for (int wi = 0; wi < cs::TUNE_WIDTHS; ++wi)
        for (int b = 0; b < cs::TUNE_SIZES; ++b) {
            const uint32_t e = cs::g_table[wi][b].load(std::memory_order_relaxed);
            if (e) std::fprintf(f, "%u %d %u %u\n", 1u << wi, b, e & 0xffu, 1u << ((e >> 8) & 0xffu));
        }
    const bool ok = std::fclose(f) == 0;
    return ok ? CS_SUCCESS : CS_ERR_INVALID_VALUE;
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
