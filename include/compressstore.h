/*
 * compressstore.h — C ABI of the B200 (sm_100a) bitmask stream-compaction library.
 *
 * Operation ("compress-store"): given a payload column T[n] and a packed bitmask of n
 * bits, write the selected elements contiguously and in order, and report how many
 * were selected.
 *
 *   mask layout : uint32 words, LSB-first. Bit (i % 32) of word (i / 32) selects
 *                 element i. ceil(n/32) words are read; bits at positions >= n are
 *                 ignored (they need not be zero).
 *   elements    : elem_bytes in {1, 2, 4, 8}; payload bits are copied verbatim
 *                 (floats are moved as their bit patterns).
 *   output      : d_out must hold at least count elements; nothing past d_out[count)
 *                 is written.
 *   count       : written to device memory (*d_count, uint64) in stream order.
 *   streams     : every call is stream-ordered and asynchronous; no call synchronizes
 *                 the stream unless its name says so.
 *   errors      : every entry point returns a cs_status (0 or negative) and never
 *                 exits the process.
 *
 * Reference interface being replaced (RememberOfLife/gpu_compressstore2):
 *   The reference has no library API. Its operator API is the header-only template
 *   family bench1..bench10 in src/benchmarks.cuh:153-440, built from the launchers
 *   launch_3pass_popc_none (src/kernels/kernel_3pass.cuh:40), launch_cub_pss
 *   (src/cub_wraps.cuh:52), launch_3pass_pss_gmem (src/kernels/kernel_3pass.cuh:107),
 *   launch_3pass_proc_true (src/kernels/kernel_3pass.cuh:536) and the scratch owner
 *   intermediate_data (src/benchmarks.cuh:53-151). The reference packs its mask
 *   MSB-first within each byte (src/data_generator.cuh:175-179); this ABI is
 *   LSB-first within uint32 words, which selects the same elements as the reference
 *   fed the per-byte bit-reversed mask.
 */
#ifndef COMPRESSSTORE_H
#define COMPRESSSTORE_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CS_API __attribute__((visibility("default")))
#else
#define CS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* cudaStream_t without pulling in the CUDA headers (same underlying type). */
typedef struct CUstream_st* cs_stream_t;

typedef enum cs_status {
    CS_PENDING = 1,              /* serving: the request has not completed yet (not an error) */
    CS_SUCCESS = 0,
    CS_ERR_INVALID_VALUE = -1,   /* bad elem_bytes, null pointer with n > 0, bad chunk length */
    CS_ERR_MISALIGNED = -2,      /* pointer not aligned as the chosen algorithm requires */
    CS_ERR_WORKSPACE = -3,       /* workspace missing, too small or not initialised */
    CS_ERR_CUDA = -4,            /* a CUDA runtime call or kernel launch failed */
    CS_ERR_TIMEOUT = -5,         /* a bounded device-side wait gave up (look-back / pipeline) */
    CS_ERR_NO_DEVICE = -6,       /* no usable sm_100 device */
    CS_ERR_OUT_OF_MEMORY = -7,   /* device allocation failed */
    CS_ERR_NOT_SUPPORTED = -8,   /* size or option outside what this build handles */
    CS_ERR_ADMISSION = -9        /* serving: request exceeds the memory budget */
} cs_status;

/* Algorithm selection. */
typedef enum cs_algo {
    CS_ALGO_AUTO = 0,   /* autotuner table (size x width bucket) */
    CS_ALGO_1PASS = 1,  /* single-pass decoupled look-back, TMA-staged persistent kernel */
    CS_ALGO_3PASS = 2,  /* chunk popcount -> chunk prefix sum -> TMA-staged writeout */
    CS_ALGO_NAIVE = 3   /* chunk popcount -> prefix sum -> warp-per-word writeout, no
                           alignment requirement beyond elem_bytes */
} cs_algo;

/* Tuning knobs. Zero-initialise and set what you need; zero means "default". */
typedef struct cs_config {
    int32_t algo;            /* cs_algo */
    uint32_t chunk_length;   /* 3-pass/naive popcount granularity in elements: power of two,
                                32 <= L <= 65536 (reference option -c/-k, main.cu:236-245).
                                0 -> 1024 */
    uint32_t grid_dim;       /* CTAs of the writeout/persistent kernel; 0 -> one wave of
                                resident CTAs (SM count x occupancy) */
    uint32_t skip;           /* 0 -> default (on), 1 -> skip payload loads of empty
                                segments, 2 -> always load whole tiles */
    uint64_t timeout_ns;     /* bound on every device-side wait; 0 -> 2 s */
    float selectivity;       /* fraction of elements the caller expects selected, in (0, 1]
                                (a query planner's estimate, say); 0 -> unknown. Under
                                CS_ALGO_AUTO a stated fraction picks the tuning table's entry
                                for its selectivity bucket (cs_tune_sel_set), where there is
                                one. The entries are measured on masks whose selected elements
                                are spread out; leave it 0 for a mask that selects long runs
                                between long empty stretches, which the default 3-pass hybrid
                                skips. Only the speed depends on it, never the result. */
} cs_config;

/* Sentinel written to *d_count when a bounded device wait gave up. */
#define CS_COUNT_ERROR 0xFFFFFFFFFFFFFFFFull

/* ------------------------------------------------------------------------------------
 * Plain call. Replaces the reference's per-call composition bench10
 * (src/benchmarks.cuh:418-440: popc -> CUB scan -> optimized writeout) and bench8
 * (src/benchmarks.cuh:384-394: cub::DeviceSelect::Flagged) as one entry point.
 * Scratch comes from a per-(device, stream) cache owned by the library, grown with
 * stream-ordered allocations (the role of intermediate_data, src/benchmarks.cuh:53-108).
 * Requires d_in, d_out 16-byte aligned and d_mask 16-byte aligned for the TMA path; other
 * element-aligned pointers are routed to CS_ALGO_NAIVE automatically.
 * ---------------------------------------------------------------------------------- */
CS_API int compressstore(const void* d_in, const void* d_mask, void* d_out, uint64_t n,
                  uint32_t elem_bytes, uint64_t* d_count, cs_stream_t stream);

/* Plain call with tuning knobs (cfg may be NULL). Same scratch cache as compressstore. */
CS_API int compressstore_cfg(const void* d_in, const void* d_mask, void* d_out, uint64_t n,
                      uint32_t elem_bytes, uint64_t* d_count, const cs_config* cfg,
                      cs_stream_t stream);

/* Allocation-free plain call (no counterpart in the reference). For callers that may not
 * allocate device memory themselves — e.g. code inside a host application whose device
 * memory is all owned by its own pool, or a loop that cannot take an allocation's implicit
 * synchronisation. Same operation and arguments as compressstore, but the scratch is a
 * fixed array of CS_NOALLOC_SCRATCH_BYTES (4 MiB) compiled into the library (held by every
 * GPU that loads it until exit), so no cudaMalloc/cudaFree or allocating library routine is
 * ever called.
 *   - n must be <= CS_NOALLOC_MAX_N (2^30) elements, any elem_bytes; larger n returns
 *     CS_ERR_NOT_SUPPORTED. The chunk length is fixed at 4096 (the tuning table still picks
 *     the algorithm), which keeps the scratch layout within the array for every such n.
 *   - The first call on a device looks the array up and zeroes it on `stream` (two small
 *     kernels); make that first call before any stream capture. The same happens again
 *     after a cudaDeviceReset, since the array then has a new address.
 *   - All calls on a device share the array; calls that overlap on the GPU (e.g. on two
 *     streams at once) race and must not be made. Nothing has to be cleared between calls. */
#define CS_NOALLOC_SCRATCH_BYTES (4u << 20)
#define CS_NOALLOC_MAX_N (1ull << 30)
CS_API int compressstore_noalloc(const void* d_in, const void* d_mask, void* d_out, uint64_t n,
                                 uint32_t elem_bytes, uint64_t* d_count, cs_stream_t stream);

/* Bytes of workspace compressstore_ex needs for (n, elem_bytes, cfg). */
CS_API size_t compressstore_workspace_size(uint64_t n, uint32_t elem_bytes, const cs_config* cfg);

/* Prepare a caller-owned workspace of ws_bytes (zero it and write its header), in stream
 * order. Must be called once before the first compressstore_ex on that workspace.
 * A workspace serves one call at a time: calls sharing it must be stream-ordered. */
CS_API int cs_workspace_init(void* d_ws, size_t ws_bytes, cs_stream_t stream);

/* Explicit-workspace call (the reference's benchN(intermediate_data*, ...) shape,
 * src/benchmarks.cuh:153-440). d_ws must have been prepared by cs_workspace_init. */
CS_API int compressstore_ex(const void* d_in, const void* d_mask, void* d_out, uint64_t n,
                     uint32_t elem_bytes, uint64_t* d_count, void* d_ws, size_t ws_bytes,
                     const cs_config* cfg, cs_stream_t stream);

/* Host-buffer call: h_in, h_mask (LSB-first uint32 words) and h_out in HOST memory; *h_count
 * receives the count. The column is streamed through the current device in 32 MB pieces
 * on internal streams: host->device copies of later pieces overlap the compaction of the
 * current piece and the device->host copy of earlier pieces' selected elements (page-locked
 * host buffers give full overlap; pageable ones work, slower). Synchronous: returns when
 * h_out[0, count) and *h_count are written. cfg may be NULL. One call at a time per device
 * (calls from several threads are serialised). The reference's driver moves whole columns
 * with synchronous copies (src/utils.cuh:41-48, src/main.cu:84-127). */
CS_API int compressstore_host(const void* h_in, const void* h_mask, void* h_out, uint64_t n, uint32_t elem_bytes,
                              uint64_t* h_count, const cs_config* cfg);
/* Free the current device's state of compressstore_host (three streams, three 32 MB piece
 * slots per direction, pinned count words: about 200 MB of device memory, kept from the
 * first call on a device until this call or process exit); a later call sets it up again.
 * Must not race with a compressstore_host call on the same device from another thread. */
CS_API int compressstore_host_release(void);

/* Synchronise the stream and report a device-side error recorded in the workspace
 * (CS_ERR_TIMEOUT after a bounded wait gave up), then clear it. */
CS_API int cs_workspace_check(void* d_ws, cs_stream_t stream);

/* Synchronise the stream and report/clear a device-side error recorded in the
 * library-owned workspace that compressstore / compressstore_cfg use on this stream. */
CS_API int compressstore_check(cs_stream_t stream);
/* Free the library-owned scratch that compressstore, compressstore_cfg and compressstore_if
 * keep for (current device, stream), in the stream's order. The library keeps one such
 * workspace per stream it has seen (up to ~1.25x the largest column's need, about 0.4% of
 * its payload) until this call or process exit; call it before destroying a stream. */
CS_API int compressstore_release(cs_stream_t stream);

/* ------------------------------------------------------------------------------------
 * The three passes as separate entry points (3-pass form).
 * ---------------------------------------------------------------------------------- */

/* Pass 1: per-chunk popcount. d_chunk_counts[c] = number of selected elements in
 * [c*L, min((c+1)*L, n)), for c < ceil(n/L). Replaces launch_3pass_popc_none /
 * kernel_3pass_popc_none_striding (src/kernels/kernel_3pass.cuh:12-57). */
CS_API int cs_popc_chunks(const uint32_t* d_mask, uint64_t n, uint32_t chunk_length,
                   uint32_t* d_chunk_counts, cs_stream_t stream);

/* Pass 2: exclusive prefix sum of chunk counts (single-pass decoupled look-back scan).
 * d_chunk_offsets[c] = sum of d_chunk_counts[0..c); *d_total = sum of all (may be NULL).
 * Replaces launch_cub_pss (src/cub_wraps.cuh:52-79), the inline
 * cub::DeviceScan::ExclusiveSum + kernel_3pass_pssskip pairs (src/benchmarks.cuh:306-309,
 * 372-375, 430-433) and launch_3pass_pss_gmem / launch_3pass_pss2_gmem
 * (src/kernels/kernel_3pass.cuh:59-214). Workspace from compressstore_workspace_size
 * or cs_scan_workspace_size, prepared by cs_workspace_init. */
CS_API size_t cs_scan_workspace_size(uint64_t chunk_count);
CS_API int cs_chunk_prefix_sum(const uint32_t* d_chunk_counts, uint64_t chunk_count,
                        uint64_t* d_chunk_offsets, uint64_t* d_total, void* d_ws,
                        size_t ws_bytes, cs_stream_t stream);

/* Pass 3: writeout. Uses the chunk offsets of pass 2 (and the chunk counts of pass 1 to
 * skip empty chunks). chunk_length must equal the one used in pass 1.
 * Replaces launch_3pass_proc_true<T, true> / kernel_3pass_proc_true_striding_optimized_
 * writeout (src/kernels/kernel_3pass.cuh:329-576) and launch_3pass_proc_none
 * (src/kernels/kernel_3pass.cuh:578-693). algo CS_ALGO_3PASS (TMA-staged, 16-byte
 * aligned pointers, chunk_length <= 4 * cs_tile_elems(elem_bytes)) or CS_ALGO_NAIVE (any
 * element-aligned pointers, any chunk length). */
CS_API int cs_writeout(const void* d_in, const uint32_t* d_mask, void* d_out, uint64_t n,
                uint32_t elem_bytes, const uint64_t* d_chunk_offsets,
                const uint32_t* d_chunk_counts, uint32_t chunk_length, int32_t algo,
                cs_stream_t stream);

/* ------------------------------------------------------------------------------------
 * Pattern compaction: the selection is a period of pattern_length (1..32) elements instead
 * of a mask in memory. Element i is selected when bit (i % pattern_length) of `pattern` is
 * set (LSB-first, like the mask words; bits >= pattern_length are ignored). No mask is read
 * and no scan runs: the count is (n / L) * popc + popc of the partial period, and every
 * output's source index has a closed form. Pointers need only element alignment (a 16-byte
 * aligned d_out gets 16-byte stores). A zero pattern writes count 0 and nothing else.
 * Replaces bench9_pattern (src/benchmarks.cuh:397-416) / launch_pattern_proc
 * (src/kernels/kernel_pattern.cuh:83-131), whose pattern starts at the most significant bit
 * (element i <-> bit 31 - i % L): pass the bit-reversed word (__brev / rev32) of such a pattern.
 * ---------------------------------------------------------------------------------- */
CS_API int compressstore_pattern(const void* d_in, void* d_out, uint64_t n, uint32_t elem_bytes,
                                 uint32_t pattern, uint32_t pattern_length, uint64_t* d_count,
                                 cs_stream_t stream);

/* ------------------------------------------------------------------------------------
 * Predicate compaction: the selection is a comparison evaluated on the payload itself on the
 * device, so no mask has to be built on the host and copied in. Element i is selected when
 * pred(d_in[i]) holds, with the elements compared as `type` (which also fixes the width).
 * The mask of the selection (LSB-first words) is written to d_mask_out when it is not NULL
 * (ceil(n/32) words, 16-byte aligned) and to library-owned scratch otherwise; the selected
 * elements are then compacted by the 3-pass writeout. Comparisons follow C++ semantics:
 * with floats, every ordered comparison with a NaN is false and NE is true.
 * d_in and d_out must be 16-byte aligned. Errors are reported as for compressstore
 * (compressstore_check on the stream). Reference: the reference evaluates its predicate on
 * the host while packing the mask (gen_predicate, src/utils.cuh:102-122; predicate
 * x > threshold, src/main.cu:24-28,92) and copies the mask to the device.
 * ---------------------------------------------------------------------------------- */
typedef enum cs_pred_op {
    CS_PRED_LT = 0,      /* x <  a */
    CS_PRED_LE = 1,      /* x <= a */
    CS_PRED_GT = 2,      /* x >  a */
    CS_PRED_GE = 3,      /* x >= a */
    CS_PRED_EQ = 4,      /* x == a */
    CS_PRED_NE = 5,      /* x != a */
    CS_PRED_BETWEEN = 6  /* a <= x && x <= b */
} cs_pred_op;

typedef enum cs_elem_type {
    CS_U8 = 0, CS_U16 = 1, CS_U32 = 2, CS_U64 = 3,
    CS_I8 = 4, CS_I16 = 5, CS_I32 = 6, CS_I64 = 7,
    CS_F32 = 8, CS_F64 = 9
} cs_elem_type;

typedef struct cs_predicate {
    int32_t op;    /* cs_pred_op */
    int32_t type;  /* cs_elem_type */
    uint64_t a;    /* constant, as the bit pattern of `type` in the low bytes */
    uint64_t b;    /* upper constant of CS_PRED_BETWEEN */
} cs_predicate;

CS_API int compressstore_if(const void* d_in, void* d_out, uint64_t n, const cs_predicate* pred,
                            uint32_t* d_mask_out, uint64_t* d_count, cs_stream_t stream);

/* ------------------------------------------------------------------------------------
 * Seeded input generators (device side). Counter-based: element i depends only on
 * (seed, i), so the CPU oracle reproduces them bit for bit. They play the role of the
 * reference's mask/data generators (src/data_generator.cuh:14-167,
 * src/kernels/data_generator.cuh:12-120) with LSB-first packing.
 * ---------------------------------------------------------------------------------- */

/* Payload: element i = low (8*elem_bytes) bits of mix64(seed, i). With float_unit != 0
 * and elem_bytes 4, element i = float((mix64(seed,i) >> 40) * 2^-24), uniform in [0,1). */
CS_API int cs_gen_payload(void* d_out, uint64_t n, uint32_t elem_bytes, uint64_t seed,
                   int32_t float_unit, cs_stream_t stream);

/* Bernoulli(p) mask: bit i = (mix64(seed, i) >> 32) < floor(p * 2^32). Writes
 * ceil(n/32) words; bits >= n are zero. */
CS_API int cs_gen_mask_bernoulli(uint32_t* d_mask, uint64_t n, double p, uint64_t seed,
                          cs_stream_t stream);

/* Alternating runs: toggle_i = (mix64(seed, i) >> 32) < floor(2^32 / mean_run);
 * bit i = toggle_0 xor ... xor toggle_i. Runs of ones and zeros have geometric lengths
 * with the given mean and the overall selectivity is 0.5. d_ws: cs_scan_workspace_size
 * bytes for ceil(n/32) chunks plus 12*ceil(n/32)+16 bytes, prepared by cs_workspace_init. */
CS_API size_t cs_gen_mask_runs_workspace_size(uint64_t n);
CS_API int cs_gen_mask_runs(uint32_t* d_mask, uint64_t n, double mean_run, uint64_t seed,
                     void* d_ws, size_t ws_bytes, cs_stream_t stream);

/* Single dense block: bits [0, k) set with k = (size_t)((float)frac * (float)n), the
 * rounding of the reference's generate_mask_clustering(frac, 1, n)
 * (src/data_generator.cuh:130-167). */
CS_API int cs_gen_mask_dense_prefix(uint32_t* d_mask, uint64_t n, float frac, cs_stream_t stream);

/* Periodic mask: bit i = bit (i % pattern_length) of pattern (1 <= pattern_length <= 32),
 * the selection of compressstore_pattern as mask words; bits >= n are zero. The reference's
 * generate_mask_pattern (src/data_generator.cuh:113-128) builds it MSB-first on the host. */
CS_API int cs_gen_mask_pattern(uint32_t* d_mask, uint64_t n, uint32_t pattern, uint32_t pattern_length,
                               cs_stream_t stream);

/* ------------------------------------------------------------------------------------
 * Batched form: many columns of uneven length and element width compacted by one plan.
 * Each column takes the 3-pass hybrid (4096-element chunks) or the 1-pass form, and each
 * pass runs ONCE for all the columns that take it: one reduce-then-scan popcount + prefix
 * launch over the 3-pass columns' blocks, one sparse-gather launch over their items, one
 * persistent TMA-staged writeout launch per element width over their units (a work list
 * spread over every SM), and one 1-pass launch per element width over the 1-pass columns'
 * units (decoupled look-back confined to each column). The plan is built once
 * (descriptors, work-to-column maps and scratch live in one device allocation made by
 * cs_batch_create); cs_batch_graph captures the launches in a CUDA graph that later
 * cs_batch_run calls replay. Column pointers are fixed by the plan; their contents may
 * change between runs.
 * Form per column: cfg->algo CS_ALGO_1PASS or CS_ALGO_3PASS forces it for every column;
 * CS_ALGO_AUTO (or cfg NULL) takes the batch table's choice for the column's (width, size,
 * selectivity) bucket (cs_tune_batch_set). When that table holds a 1-pass entry,
 * cs_batch_create measures each column's selectivity with one popcount pass over the masks
 * as they are at that moment (into plan-owned memory); the choice affects speed only.
 * Reference: the reference's only multi-segment form is the 2-stream split with offset
 * stitching of bench3_3pass_streaming (src/benchmarks.cuh:195-293,
 * src/kernels/kernel_streaming_add.cuh:8-16).
 * ---------------------------------------------------------------------------------- */
typedef struct cs_column {
    const void* d_in;     /* 16-byte aligned */
    const void* d_mask;   /* 16-byte aligned, LSB-first uint32 words */
    void* d_out;          /* 16-byte aligned, room for the column's count */
    uint64_t n;
    uint32_t elem_bytes;  /* 1, 2, 4 or 8 */
    uint32_t reserved;
    uint64_t* d_count;    /* 8-byte aligned device word */
} cs_column;

typedef struct cs_batch cs_batch;

/* Build a plan for ncols columns (copied). Allocates the plan's device memory and uploads
 * its descriptors (synchronises the stream). cfg may be NULL (timeout_ns is honoured). */
CS_API int cs_batch_create(cs_batch** out, const cs_column* cols, uint32_t ncols, const cs_config* cfg,
                           cs_stream_t stream);
/* Run the plan on the stream (replays the captured graph when there is one). */
CS_API int cs_batch_run(cs_batch* b, cs_stream_t stream);
/* Capture the plan's launches in a CUDA graph; later cs_batch_run calls launch the graph. */
CS_API int cs_batch_graph(cs_batch* b, cs_stream_t stream);
/* Synchronise the stream and report a device-side error of the plan's runs (then clear it). */
CS_API int cs_batch_check(cs_batch* b, cs_stream_t stream);
/* Device bytes held by the plan. */
CS_API uint64_t cs_batch_device_bytes(const cs_batch* b);
/* Kernel launches one cs_batch_run issues (1 when a graph is replayed). */
CS_API uint32_t cs_batch_launches(const cs_batch* b);
/* Columns of the plan that take the 1-pass form. */
CS_API uint32_t cs_batch_one_pass_columns(const cs_batch* b);
/* The per-call baseline the plan replaces: one plain compressstore per column, in column
 * order, on the stream (library-owned scratch); same outputs as cs_batch_run. */
CS_API int cs_batch_run_per_call(cs_batch* b, cs_stream_t stream);
CS_API int cs_batch_destroy(cs_batch* b);

/* ------------------------------------------------------------------------------------
 * Serving loop: compaction requests over device-resident payloads and masks, admitted by
 * an output-memory budget and batched as they arrive (continuous batching).
 *
 * A request names a payload column and its mask already in device memory (the caller's
 * resident pool) and gets its output from the server's arena: on admission it reserves
 * n * elem_bytes bytes (the most it can select), which shrink to count * elem_bytes when
 * it completes and return to the arena on cs_server_release. Requests wait, in arrival
 * order, until the arena can hold them. A scheduler thread forms a batch from every
 * admitted request not yet running (up to max_batch requests and max_batch_elems
 * elements) as soon as one of `slots` batch slots is free, and launches it as one
 * multi-column plan (the batched form's three launches: fused popcount+scan, sparse
 * gather, TMA writeout per width) on that slot's stream. Up to `slots` batches are on the
 * GPU at once, so requests that arrive while others run are launched beside them instead
 * of waiting for them. A request's output is the same whichever batch it lands in.
 * CS_SERVE_PER_CALL runs each admitted request as its own compressstore_ex call (the
 * per-call baseline) with the same admission, slots and bookkeeping.
 * The reference has no serving form; its only overlap of independent work is the 2-stream
 * split of bench3_3pass_streaming (src/benchmarks.cuh:195-293).
 * ---------------------------------------------------------------------------------- */
typedef enum cs_serve_mode {
    CS_SERVE_BATCH = 0,     /* continuous batching: one multi-column plan per batch */
    CS_SERVE_PER_CALL = 1   /* one compressstore_ex call per request */
} cs_serve_mode;

typedef struct cs_server_config {
    uint64_t out_budget_bytes; /* output arena; 0 -> min(4 GiB, a quarter of free memory) */
    uint64_t max_batch_elems;  /* elements per batch and largest request; 0 -> 2^28 */
    uint32_t max_batch;        /* requests per batch; 0 -> 64 */
    uint32_t slots;            /* batches in flight; 0 -> 3 */
    int32_t mode;              /* cs_serve_mode */
    uint32_t reserved;
    uint64_t timeout_ns;       /* bound on device-side waits; 0 -> 2 s */
} cs_server_config;

typedef struct cs_request {
    const void* d_in;     /* device payload, 16-byte aligned; must stay valid until completion */
    const void* d_mask;   /* device LSB-first uint32 mask words, 16-byte aligned */
    uint64_t n;           /* elements, 0 <= n <= max_batch_elems */
    uint32_t elem_bytes;  /* 1, 2, 4 or 8 */
    uint32_t reserved;
} cs_request;

typedef struct cs_result {
    void* d_out;          /* selected elements in the server's arena (valid until release) */
    uint64_t count;       /* selected elements */
    uint64_t latency_ns;  /* submit -> results visible to the host */
    uint64_t queue_ns;    /* submit -> launch of its batch */
    int32_t status;       /* cs_status of the request */
    uint32_t batch_size;  /* requests in the batch it ran in */
} cs_result;

typedef struct cs_server_stats {
    uint64_t submitted, completed, rejected;
    uint64_t batches;          /* batches (or per-call launches) issued */
    uint64_t batched_requests; /* sum of batch sizes */
    uint64_t arena_bytes, arena_used, arena_peak;
    uint64_t kernel_launches;  /* kernels launched by the server's scheduler */
} cs_server_stats;

typedef struct cs_server cs_server;

/* Create a server on the current device (allocates its arena and slot buffers and
 * starts its scheduler thread). cfg may be NULL. */
CS_API int cs_server_create(cs_server** out, const cs_server_config* cfg);
/* Queue a request; *ticket identifies it. Returns CS_ERR_ADMISSION if it can never fit
 * the arena, CS_ERR_NOT_SUPPORTED if n > max_batch_elems, CS_ERR_MISALIGNED /
 * CS_ERR_INVALID_VALUE for bad pointers or widths. Thread-safe. */
CS_API int cs_server_submit(cs_server* s, const cs_request* req, uint64_t* ticket);
/* CS_SUCCESS with *res filled once the request completed (res->status carries its own
 * outcome), CS_PENDING before, CS_ERR_INVALID_VALUE for an unknown ticket. */
CS_API int cs_server_poll(cs_server* s, uint64_t ticket, cs_result* res);
/* As cs_server_poll, blocking up to timeout_ns (0: no limit); CS_PENDING if it ran out. */
CS_API int cs_server_wait(cs_server* s, uint64_t ticket, uint64_t timeout_ns, cs_result* res);
/* The next completed request not yet returned by this call (any order of completion),
 * blocking up to timeout_ns (0: no limit); CS_PENDING if none completed in time. */
CS_API int cs_server_next(cs_server* s, uint64_t timeout_ns, uint64_t* ticket, cs_result* res);
/* Return a completed request's output space to the arena and forget the ticket. */
CS_API int cs_server_release(cs_server* s, uint64_t ticket);
CS_API int cs_server_stats_get(cs_server* s, cs_server_stats* st);
/* Load generator: submit reqs[i] at arrival_ns[i] after the call starts (non-decreasing
 * offsets, e.g. Poisson arrivals), take each completion as it comes, copy it to
 * results[i] and release it (results[i].d_out is then NULL). Returns when all completed.
 * The server must have no other outstanding requests. */
CS_API int cs_server_replay(cs_server* s, const cs_request* reqs, const uint64_t* arrival_ns, uint32_t count,
                            cs_result* results);
/* Wait for every launched batch, stop the scheduler and free the server's memory. */
CS_API int cs_server_destroy(cs_server* s);

/* ------------------------------------------------------------------------------------
 * Autotuner table for CS_ALGO_AUTO. The reference picks chunk length, block and grid by
 * an exhaustive sweep per run (src/main.cu:168-190) and keeps the fastest per phase in
 * SQL views (eval/eval.db); here the project's autotuner measures once and installs one
 * choice per (element width, size bucket) with cs_tune_set.
 * size_bucket = floor(log2(n)) / 2, clamped to [0, 20]. algo CS_ALGO_AUTO clears it.
 * ---------------------------------------------------------------------------------- */
CS_API int cs_tune_set(uint32_t elem_bytes, int32_t size_bucket, int32_t algo, uint32_t chunk_length);
/* Install a table written by the autotuner (text, one "elem_bytes size_bucket algo
 * chunk_length" entry per line, '#' comments); all lines are validated first. A table named
 * by the environment variable CS_TUNE_TABLE is installed before the first lookup.
 * cs_tune_save writes the installed entries in the same format. */
CS_API int cs_tune_load(const char* path);
CS_API int cs_tune_save(const char* path);
CS_API int cs_tune_get(uint32_t elem_bytes, uint64_t n, int32_t* algo, uint32_t* chunk_length);
CS_API int cs_tune_size_bucket(uint64_t n);
/* Plain call with a stated selectivity (cs_config.selectivity > 0): the choice per
 * (element width, size bucket, selectivity bucket), sel_bucket = cs_tune_sel_bucket(fraction);
 * algo CS_ALGO_AUTO clears an entry. Where none is set the (width, size) entry above
 * applies. The plain call cannot measure the selectivity before it runs without a pass of
 * its own, so only a caller who knows it gets this choice; the batched form measures it when
 * a plan is built. In table files these are the lines
 * "sel elem_bytes size_bucket sel_bucket algo chunk_length". cs_tune_sel_get returns what
 * CS_ALGO_AUTO takes for that n and fraction (0 = unknown). */
CS_API int cs_tune_sel_set(uint32_t elem_bytes, int32_t size_bucket, int32_t sel_bucket, int32_t algo,
                           uint32_t chunk_length);
CS_API int cs_tune_sel_get(uint32_t elem_bytes, uint64_t n, double selectivity, int32_t* algo,
                           uint32_t* chunk_length);
/* Batched form's table: the algorithm (CS_ALGO_1PASS or CS_ALGO_3PASS) a column takes inside
 * a plan built with CS_ALGO_AUTO, per (element width, size bucket, selectivity bucket);
 * sel_bucket = cs_tune_sel_bucket(fraction selected): [0, 0.05) -> 0, [0.05, 0.3) -> 1,
 * [0.3, 0.7] -> 2, (0.7, 0.95] -> 3, (0.95, 1] -> 4. Unset entries (and algo CS_ALGO_AUTO, which clears one) mean 3-pass. In
 * table files these are the lines "batch elem_bytes size_bucket sel_bucket algo". The
 * reference's analogue is again its sweep (src/main.cu:168-190). */
CS_API int cs_tune_batch_set(uint32_t elem_bytes, int32_t size_bucket, int32_t sel_bucket, int32_t algo);
CS_API int cs_tune_batch_get(uint32_t elem_bytes, uint64_t n, double selectivity, int32_t* algo);
CS_API int cs_tune_sel_bucket(double selectivity);

/* ------------------------------------------------------------------------------------
 * Library info.
 * ---------------------------------------------------------------------------------- */
CS_API const char* cs_status_string(int status);
/* Number of kernel launches issued by this library in the calling process (all threads). */
CS_API uint64_t cs_launch_count(void);
/* Tile size (elements) of the TMA-staged kernels for elem_bytes; their look-back unit and
 * 3-pass chunk-length limit is 4 tiles. */
CS_API uint32_t cs_tile_elems(uint32_t elem_bytes);

/* Dynamic shared memory in bytes of one CTA of the TMA-staged persistent kernel for
 * elem_bytes and algo (CS_ALGO_1PASS or CS_ALGO_3PASS); 0 for other arguments. Diagnostic. */
CS_API uint32_t cs_compact_smem_bytes(uint32_t elem_bytes, int32_t algo);
/* Library version as 0xMMmmpp. */
CS_API uint32_t cs_version(void);

#ifdef __cplusplus
}
#endif

#endif /* COMPRESSSTORE_H */
