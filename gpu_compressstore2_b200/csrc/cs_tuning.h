// cs_tuning.h — algorithm choice for CS_ALGO_AUTO, keyed by size and element-width
// bucket (and, where the caller states it or the batched form measures it, selectivity). The table is the output of the project's autotuner (it replaces the
// reference's brute-force chunk x block x grid sweep, src/main.cu:168-190, and the
// min-per-phase views of eval/eval.db); cs_tune_set overrides an entry at run time.
#pragma once
#include <cstdint>

namespace cs {

struct TuneChoice {
    int algo;              // cs_algo (never CS_ALGO_AUTO)
    uint32_t chunk_length; // 3-pass popcount granularity
};

// Buckets: elem width index (1,2,4,8 bytes -> 0..3) x size bucket floor(log2(n)) / 2
// clamped to [0, 20].
constexpr int TUNE_WIDTHS = 4;
constexpr int TUNE_SIZES = 21;

int tune_size_bucket(uint64_t n);
int tune_width_index(uint32_t elem_bytes);

// Batched form: the algorithm (CS_ALGO_1PASS or CS_ALGO_3PASS) of a column inside a plan,
// keyed by element width, size bucket and selectivity bucket (the fraction selected, measured
// when the plan is built). Inside a plan the passes are shared by every column, so the choice
// weighs mask traffic and look-back waits, not launch latency as in the plain call's table.
constexpr int TUNE_SELS = 5;
// [0, 0.05) -> 0, [0.05, 0.3) -> 1, [0.3, 0.7] -> 2, (0.7, 0.95] -> 3, (0.95, 1] -> 4
int tune_sel_bucket(double selectivity);
int tune_batch_lookup(uint64_t n, uint32_t elem_bytes, double selectivity); // CS_ALGO_3PASS if unset
bool tune_batch_any_1pass();                         // some entry picks the 1-pass form

// Plain call: the choice for (width, size bucket). A caller that knows the fraction it
// expects selected passes it (selectivity in (0, 1]; 0 = unknown): the entry of its
// selectivity bucket is taken when the table has one, the (width, size) entry otherwise.
TuneChoice tune_lookup(uint64_t n, uint32_t elem_bytes, double selectivity = 0.0);

} // namespace cs
