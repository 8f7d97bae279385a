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
// Batched form: algo per (width, size bucket, selectivity bucket). Zero = unset (3-pass).
std::atomic<uint32_t> g_batch[TUNE_WIDTHS][TUNE_SIZES][TUNE_SELS];
// Plain call with a stated selectivity: packed like g_table. Zero = unset (use g_table).
std::atomic<uint32_t> g_sel[TUNE_WIDTHS][TUNE_SIZES][TUNE_SELS];

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

// Five buckets: on B200 the faster form changes twice between p = 0.05 and 0.95 (at 2^28
// f32 the 1-pass wins at p = 0.1 and 0.9, the 3-pass at 0.5), which one middle bucket
// sampled at 0.5 could not follow.
int tune_sel_bucket(double selectivity)
{
    if (!(selectivity >= 0.05)) return 0;
    if (selectivity < 0.3) return 1;
    if (selectivity <= 0.7) return 2;
    if (selectivity <= 0.95) return 3;
    return 4;
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

// Packed (algo, chunk length) of a plain-call entry; 0 for CS_ALGO_AUTO (clear), UINT32_MAX
// for invalid arguments.
uint32_t pack_choice(int32_t algo, uint32_t chunk_length)
{
    if (algo == CS_ALGO_AUTO) return 0u;
    if (algo < CS_ALGO_1PASS || algo > CS_ALGO_NAIVE) return UINT32_MAX;
    if (chunk_length < 32 || chunk_length > 65536 || (chunk_length & (chunk_length - 1))) return UINT32_MAX;
    uint32_t lg = 0;
    while ((1u << lg) < chunk_length) ++lg;
    return static_cast<uint32_t>(algo) | (lg << 8);
}

int set_entry(uint32_t elem_bytes, int32_t size_bucket, int32_t algo, uint32_t chunk_length)
{
    const int wi = tune_width_index(elem_bytes);
    if (wi < 0 || size_bucket < 0 || size_bucket >= TUNE_SIZES) return CS_ERR_INVALID_VALUE;
    const uint32_t e = pack_choice(algo, chunk_length);
    if (e == UINT32_MAX) return CS_ERR_INVALID_VALUE;
    g_table[wi][size_bucket].store(e);
    return CS_SUCCESS;
}

int set_sel_entry(uint32_t elem_bytes, int32_t size_bucket, int32_t sel_bucket, int32_t algo, uint32_t chunk_length)
{
    const int wi = tune_width_index(elem_bytes);
    if (wi < 0 || size_bucket < 0 || size_bucket >= TUNE_SIZES || sel_bucket < 0 || sel_bucket >= TUNE_SELS)
        return CS_ERR_INVALID_VALUE;
    const uint32_t e = pack_choice(algo, chunk_length);
    if (e == UINT32_MAX) return CS_ERR_INVALID_VALUE;
    g_sel[wi][size_bucket][sel_bucket].store(e);
    return CS_SUCCESS;
}

int set_batch_entry(uint32_t elem_bytes, int32_t size_bucket, int32_t sel_bucket, int32_t algo)
{
    const int wi = tune_width_index(elem_bytes);
    if (wi < 0 || size_bucket < 0 || size_bucket >= TUNE_SIZES || sel_bucket < 0 || sel_bucket >= TUNE_SELS)
        return CS_ERR_INVALID_VALUE;
    if (algo != CS_ALGO_AUTO && algo != CS_ALGO_1PASS && algo != CS_ALGO_3PASS) return CS_ERR_INVALID_VALUE;
    g_batch[wi][size_bucket][sel_bucket].store(static_cast<uint32_t>(algo));
    return CS_SUCCESS;
}

// Text table, '#' starts a comment; every line is validated before any entry is installed:
//   "elem_bytes size_bucket algo chunk_length"                plain call (CS_ALGO_AUTO)
//   "sel elem_bytes size_bucket sel_bucket algo chunk_length" plain call, stated selectivity
//   "batch elem_bytes size_bucket sel_bucket algo"            batched form
int load_table_file(const char* path)
{
    FILE* f = std::fopen(path, "r");
    if (!f) return CS_ERR_INVALID_VALUE;
    enum Kind { PLAIN, SEL, BATCH };
    struct Entry {
        Kind kind;
        uint32_t w;
        int32_t b, s, a;
        uint32_t c;
    };
    constexpr int MAX_ENTRIES = TUNE_WIDTHS * TUNE_SIZES * (1 + 2 * TUNE_SELS);
    static thread_local Entry entries[MAX_ENTRIES];
    int count = 0, rc = CS_SUCCESS;
    char line[256];
    while (std::fgets(line, sizeof(line), f)) {
        char* hash = line;
        while (*hash && *hash != '#') ++hash;
        *hash = 0;
        unsigned w = 0, c = 0;
        int b = 0, a = 0, sb = 0;
        char extra = 0;
        Entry e{};
        bool ok;
        const int gotb = std::sscanf(line, " batch %u %d %d %d %c", &w, &b, &sb, &a, &extra);
        const int gots = gotb > 0 ? 0 : std::sscanf(line, " sel %u %d %d %d %u %c", &w, &b, &sb, &a, &c, &extra);
        if (gotb > 0) {
            ok = gotb == 4 && tune_width_index(w) >= 0 && b >= 0 && b < TUNE_SIZES && sb >= 0 && sb < TUNE_SELS &&
                 (a == CS_ALGO_AUTO || a == CS_ALGO_1PASS || a == CS_ALGO_3PASS);
            e = Entry{BATCH, w, b, sb, a, 0};
        } else if (gots > 0) {
            ok = gots == 5 && tune_width_index(w) >= 0 && b >= 0 && b < TUNE_SIZES && sb >= 0 && sb < TUNE_SELS &&
                 pack_choice(a, c) != UINT32_MAX;
            e = Entry{SEL, w, b, sb, a, c};
        } else {
            const int got = std::sscanf(line, " %u %d %d %u %c", &w, &b, &a, &c, &extra);
            if (got <= 0) {
                // blank or comment line, unless it holds something that is not an entry
                char word[8] = {0};
                if (std::sscanf(line, " %7s", word) <= 0) continue;
                ok = false;
            } else {
                ok = got == 4 && tune_width_index(w) >= 0 && b >= 0 && b < TUNE_SIZES && a >= CS_ALGO_AUTO &&
                     a <= CS_ALGO_NAIVE && (a == CS_ALGO_AUTO || (c >= 32 && c <= 65536 && !(c & (c - 1))));
            }
            e = Entry{PLAIN, w, b, 0, a, c};
        }
        if (!ok || count == MAX_ENTRIES) {
            rc = CS_ERR_INVALID_VALUE;
            break;
        }
        entries[count++] = e;
    }
    std::fclose(f);
    if (rc != CS_SUCCESS) return rc;
    for (int i = 0; i < count; ++i) {
        const Entry& e = entries[i];
        if (e.kind == BATCH) set_batch_entry(e.w, e.b, e.s, e.a);
        else if (e.kind == SEL) set_sel_entry(e.w, e.b, e.s, e.a, e.c);
        else set_entry(e.w, e.b, e.a, e.c);
    }
    return CS_SUCCESS;
}

TuneChoice tune_lookup(uint64_t n, uint32_t elem_bytes, double selectivity)
{
    load_env_table_once();
    const int wi = tune_width_index(elem_bytes);
    if (wi < 0) return default_choice(n, elem_bytes);
    const int b = tune_size_bucket(n);
    uint32_t e = 0;
    if (selectivity > 0.0) e = g_sel[wi][b][tune_sel_bucket(selectivity)].load(std::memory_order_relaxed);
    if (e == 0) e = g_table[wi][b].load(std::memory_order_relaxed);
    if (e == 0) return default_choice(n, elem_bytes);
    return TuneChoice{static_cast<int>(e & 0xffu), 1u << ((e >> 8) & 0xffu)};
}

int tune_batch_lookup(uint64_t n, uint32_t elem_bytes, double selectivity)
{
    load_env_table_once();
    const int wi = tune_width_index(elem_bytes);
    if (wi < 0) return CS_ALGO_3PASS;
    const uint32_t e = g_batch[wi][tune_size_bucket(n)][tune_sel_bucket(selectivity)].load(std::memory_order_relaxed);
    return e == CS_ALGO_1PASS ? CS_ALGO_1PASS : CS_ALGO_3PASS;
}

bool tune_batch_any_1pass()
{
    load_env_table_once();
    for (int wi = 0; wi < TUNE_WIDTHS; ++wi)
        for (int b = 0; b < TUNE_SIZES; ++b)
            for (int s = 0; s < TUNE_SELS; ++s)
                if (g_batch[wi][b][s].load(std::memory_order_relaxed) == CS_ALGO_1PASS) return true;
    return false;
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
    std::fprintf(f, "# sel elem_bytes size_bucket sel_bucket algo chunk_length  (plain call with a stated "
                    "selectivity; sel_bucket: selected fraction [0,0.05) 0, [0.05,0.3) 1, [0.3,0.7] 2, "
                    "(0.7,0.95] 3, (0.95,1] 4)\n");
    for (int wi = 0; wi < cs::TUNE_WIDTHS; ++wi)
        for (int b = 0; b < cs::TUNE_SIZES; ++b)
            for (int sb = 0; sb < cs::TUNE_SELS; ++sb) {
                const uint32_t e = cs::g_sel[wi][b][sb].load(std::memory_order_relaxed);
                if (e) std::fprintf(f, "sel %u %d %d %u %u\n", 1u << wi, b, sb, e & 0xffu, 1u << ((e >> 8) & 0xffu));
            }
    std::fprintf(f, "# batch elem_bytes size_bucket sel_bucket algo  (sel_bucket as above)\n");
    for (int wi = 0; wi < cs::TUNE_WIDTHS; ++wi)
        for (int b = 0; b < cs::TUNE_SIZES; ++b)
            for (int sb = 0; sb < cs::TUNE_SELS; ++sb) {
                const uint32_t e = cs::g_batch[wi][b][sb].load(std::memory_order_relaxed);
                if (e) std::fprintf(f, "batch %u %d %d %u\n", 1u << wi, b, sb, e);
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

int cs_tune_sel_set(uint32_t elem_bytes, int32_t size_bucket, int32_t sel_bucket, int32_t algo, uint32_t chunk_length)
{
    cs::load_env_table_once();
    return cs::set_sel_entry(elem_bytes, size_bucket, sel_bucket, algo, chunk_length);
}

int cs_tune_sel_get(uint32_t elem_bytes, uint64_t n, double selectivity, int32_t* algo, uint32_t* chunk_length)
{
    if (cs::tune_width_index(elem_bytes) < 0 || !algo || !chunk_length || !(selectivity >= 0.0 && selectivity <= 1.0))
        return CS_ERR_INVALID_VALUE;
    const cs::TuneChoice t = cs::tune_lookup(n, elem_bytes, selectivity);
    *algo = t.algo;
    *chunk_length = t.chunk_length;
    return CS_SUCCESS;
}

int cs_tune_size_bucket(uint64_t n)
{
    return cs::tune_size_bucket(n);
}

int cs_tune_batch_set(uint32_t elem_bytes, int32_t size_bucket, int32_t sel_bucket, int32_t algo)
{
    cs::load_env_table_once();
    return cs::set_batch_entry(elem_bytes, size_bucket, sel_bucket, algo);
}

int cs_tune_batch_get(uint32_t elem_bytes, uint64_t n, double selectivity, int32_t* algo)
{
    if (cs::tune_width_index(elem_bytes) < 0 || !algo) return CS_ERR_INVALID_VALUE;
    *algo = cs::tune_batch_lookup(n, elem_bytes, selectivity);
    return CS_SUCCESS;
}

int cs_tune_sel_bucket(double selectivity)
{
    return cs::tune_sel_bucket(selectivity);
}

} // extern "C"
