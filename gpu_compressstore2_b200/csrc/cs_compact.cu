// cs_compact.cu — the TMA-staged, warp-specialised persistent compaction kernel.
//
// Work is split into UNITS of U consecutive tiles; a tile is TILE_BYTES of payload
// (TILE_BYTES/w elements). One CTA per SM takes units one after another (an atomic ticket
// per unit in the 1-pass form, static round robin in the 3-pass form) and streams them
// through two shared-memory rings: a ring of unit masks (3 slots in the 3-pass form, 4 in
// the 1-pass form) and an S-stage ring of payload tiles.
//
//   warp 0  producer : takes unit j+AHEAD and issues its mask (1-D TMA bulk copy,
//                      cp.async.bulk, no multicast) BEFORE the payload tiles of unit j, so the
//                      scanner works ahead (AHEAD = 1 in the 3-pass form, 2 in the 1-pass
//                      form). For each payload tile it reads the landed mask and copies only
//                      the 1 KB segments that hold a selected element (the whole tile in one
//                      copy when all do). Ragged tails are finished with plain loads.
//   warp 1  scanner  : popcounts the unit's mask and scans it into per-tile,
//                      per-compute-warp bases. 3-pass: loads the unit's pass-2 chunk offset
//                      and publishes it. 1-pass: publishes the unit's aggregate status at
//                      once and hands the unit to the look-back warp.
//   warp 2  look-back (1-pass only): decoupled look-back over unit statuses; publishes the
//                      unit's prefix status and its output offset.
//   then    compute  : NC warps, each owning TILE_BYTES/NC contiguous bytes of every tile.
//                      Lanes read 16-byte payload vectors from shared memory and place the
//                      selected elements into a per-warp staging buffer at their output
//                      positions (popc of the mask bits below them), release the stage, then
//                      emit the staged run with 16-byte streaming stores; only the ragged
//                      head/tail vectors are written element by element.
//
// Reference: kernel_3pass_proc_true_striding_optimized_writeout
// (src/kernels/kernel_3pass.cuh:329-467) stages 32 source indices per warp and gathers
// from global memory; the popcount and prefix passes it depends on are
// src/kernels/kernel_3pass.cuh:12-214; its empty-chunk skipping is :268-288. Every wait is
// bounded (timeout_ns) and leaves the kernel through the normal exit path with an error
// recorded in the workspace header.
#include <cstdint>
#include <cuda_runtime.h>

#include "cs_internal.cuh"

// MASK_ROT: a lane reads its KWORDS mask words of a tile as 16-byte vectors starting at
// vector (lane % (KWORDS / 4)). Lane strides of KWORDS words (128 B for 1-byte elements) put
// every lane of a quarter warp on the same banks when all start at vector 0; the rotation
// spreads them (sums and ORs over the words do not depend on the order).

namespace cs {

#ifndef CS_NCW
#define CS_NCW 16
#endif
#ifndef CS_STAGES
#define CS_STAGES 4
#endif
#ifndef CS_MSLOTS
#define CS_MSLOTS 3
#endif
#ifndef CS_MSLOTS_1PASS
#define CS_MSLOTS_1PASS 4
#endif
constexpr int NCW = CS_NCW;             // compute warps
// Warp roles: 0 producer, 1 scanner, then (1-pass only) one look-back warp, then the compute
// warps. In the 1-pass form the scanner publishes each unit's aggregate as soon as the
// unit's mask has landed, and the look-back warp resolves the unit's prefix separately, so
// a scanner never holds back its next aggregate while its current look-back waits.
template <int MODE>
struct Roles {
    static constexpr int LOOKBACK = MODE == 0 ? 2 : -1;         // look-back warp (1-pass only)
    static constexpr int FIRST_COMPUTE = MODE == 0 ? 3 : 2;     // first compute warp
    static constexpr int NTHREADS = (FIRST_COMPUTE + NCW) * 32;
    // Unit masks in flight per CTA: one being consumed, MSLOTS - 2 scanned ahead, one free for
    // the producer. The 1-pass form keeps its masks two units ahead, so each unit's look-back
    // has about two units of writeout time to finish before the compute warps need its offset.
    static constexpr int MSLOTS = MODE == 0 ? CS_MSLOTS_1PASS : CS_MSLOTS;
    static constexpr uint32_t AHEAD = MSLOTS - 2; // units the producer takes beyond the one it streams
    static_assert(MSLOTS >= 3, "one unit consumed, one ahead, one free");
};
constexpr int STAGES = CS_STAGES;       // payload tiles in flight per CTA (see Kernel::S)

template <int U, int NC>
struct UnitMeta {
    int64_t unit;              // unit index of this launch; -1: end of work
    uint64_t ul;               // unit index within its column
    uint64_t prefix;           // output offset of the unit (POISON: do not write)
    uint32_t col;              // column of the unit (0 for a single column)
    uint32_t total;            // selected elements of the unit (1-pass: scanner -> look-back warp)
    uint32_t warp_base[U][NC]; // output offset of each compute warp's segment, from the unit start
};

template <typename T, int S, int NC, int MSLOTS, int UT = UNIT_TILES>
struct Layout {
    static constexpr uint32_t U = UT;
    static constexpr uint32_t TE = TILE_BYTES / sizeof(T); // tile elements
    static constexpr uint32_t W = TE / 32;                  // mask words per tile
    static constexpr uint32_t UMASK_BYTES = U * W * 4;      // mask bytes per unit
    static constexpr uint32_t SEG_BYTES = TILE_BYTES / NC;  // payload bytes per compute warp
    static constexpr uint32_t STAGE_OUT_BYTES = SEG_BYTES + 16;
    static constexpr uint32_t PAY = 0;
    static constexpr uint32_t MASK = PAY + S * TILE_BYTES;
    static constexpr uint32_t OUTB = MASK + MSLOTS * UMASK_BYTES;
    static constexpr uint32_t META = OUTB + NC * STAGE_OUT_BYTES;
    static constexpr uint32_t BARS = (META + MSLOTS * sizeof(UnitMeta<U, NC>) + 15u) & ~15u;
    static constexpr uint32_t NBARS = 2 * S + 4 * MSLOTS;
    static constexpr uint32_t TOTAL = BARS + NBARS * 8;
    static_assert(UMASK_BYTES % 16 == 0, "mask slot must keep 16-byte alignment");
    static_assert(SEG_BYTES % 16 == 0 && (TE / NC) % 32 == 0, "segments must be whole words and vectors");
    static_assert(W % 128 == 0, "scanner reads 4 words per lane step");
    static_assert(TOTAL <= 227 * 1024, "shared memory budget");
};

// ---------------------------------------------------------------------------------
// Placement of one compute warp's segment of a landed tile (PASSES passes of WPP mask
// words, 32 elements each) into the warp's stage: every selected element goes to
// stage[run + number of selected elements before it]. Each returns the new run. `seg`
// points at the segment's payload, `segm` at its mask words, both in shared memory.
// ---------------------------------------------------------------------------------

// Each lane takes one 16-byte vector (VEC elements) per 32*VEC-element group. Every
// shared-memory load and shuffle of the segment is issued before its first stage store, so
// their latencies overlap. (The stores may alias the loaded shared memory, which keeps the
// compiler from moving a later group's loads above an earlier group's stores.)
template <typename T, uint32_t PASSES, uint32_t WPP>
__device__ __forceinline__ uint32_t place_vectors(const T* seg, const uint32_t* segm, T* stage, uint32_t run,
                                                  uint32_t lane)
{
    constexpr uint32_t VEC = 16 / sizeof(T);
    constexpr uint32_t GROUPS = WPP / VEC;
    constexpr uint32_t NG = PASSES * GROUPS;
    uint32_t m[PASSES], excl[PASSES], ptot[PASSES], nzw[PASSES];
#pragma unroll
    for (uint32_t pass = 0; pass < PASSES; ++pass) m[pass] = (lane < WPP) ? segm[pass * WPP + lane] : 0u;
#pragma unroll
    for (uint32_t pass = 0; pass < PASSES; ++pass) {
        nzw[pass] = __ballot_sync(0xffffffffu, m[pass] != 0u); // non-empty words of the pass
        const uint32_t c = __popc(m[pass]);
        const uint32_t incl = warp_incl_scan(c, lane);
        excl[pass] = incl - c;
        ptot[pass] = __shfl_sync(0xffffffffu, incl, 31);
    }
    union {
        uint4 v;
        T e[VEC];
    } x[NG];
    uint32_t bits[NG], pos[NG];
    const uint32_t sh = (lane * VEC) & 31u;
#pragma unroll
    for (uint32_t pass = 0; pass < PASSES; ++pass) {
#pragma unroll
        for (uint32_t g = 0; g < GROUPS; ++g) {
            const uint32_t k = pass * GROUPS + g;
            const uint32_t src = g * VEC + lane / (32 / VEC);
            const uint32_t mw = __shfl_sync(0xffffffffu, m[pass], src);
            const uint32_t me = __shfl_sync(0xffffffffu, excl[pass], src);
            bits[k] = (mw >> sh) & ((1u << VEC) - 1u);
            pos[k] = run + me + __popc(mw & ((1u << sh) - 1u));
            x[k].v = lds128(seg + pass * WPP * 32 + g * 32 * VEC + lane * VEC);
        }
        run += ptot[pass];
    }
#pragma unroll
    for (uint32_t k = 0; k < NG; ++k) {
        const uint32_t pass = k / GROUPS, g = k % GROUPS;
        if (((nzw[pass] >> (g * VEC)) & ((VEC < 32 ? (1u << VEC) : 0u) - 1u)) == 0u) continue; // empty group (warp-uniform)
        uint32_t ps = pos[k];
#pragma unroll
        for (uint32_t e = 0; e < VEC; ++e) {
            if ((bits[k] >> e) & 1u) stage[ps] = x[k].e[e];
            ps += (bits[k] >> e) & 1u;
        }
    }
    return run;
}

// Same lane assignment, one group at a time (load, shuffles, stores). The 3-pass writeout of
// 4- and 8-byte elements measured faster this way at p = 0.5 (2.6% at 2^28 f32).
template <typename T, uint32_t PASSES, uint32_t WPP>
__device__ __forceinline__ uint32_t place_grouped(const T* seg, const uint32_t* segm, T* stage, uint32_t run,
                                                  uint32_t lane)
{
    constexpr uint32_t VEC = 16 / sizeof(T);
    constexpr uint32_t GROUPS = WPP / VEC;
#pragma unroll
    for (uint32_t pass = 0; pass < PASSES; ++pass) {
        const uint32_t m = (lane < WPP) ? segm[pass * WPP + lane] : 0u;
        const uint32_t nzw = __ballot_sync(0xffffffffu, m != 0u); // non-empty words of the pass
        if (nzw == 0u) continue;                                   // warp-uniform
        const uint32_t c = __popc(m);
        const uint32_t incl = warp_incl_scan(c, lane);
        const uint32_t excl = incl - c;
        const uint32_t pass_total = __shfl_sync(0xffffffffu, incl, 31);
#pragma unroll
        for (uint32_t g = 0; g < GROUPS; ++g) {
            if (((nzw >> (g * VEC)) & ((VEC < 32 ? (1u << VEC) : 0u) - 1u)) == 0u) continue; // empty group
            const uint32_t src = g * VEC + lane / (32 / VEC);
            const uint32_t mw = __shfl_sync(0xffffffffu, m, src);
            const uint32_t me = __shfl_sync(0xffffffffu, excl, src);
            const uint32_t sh = (lane * VEC) & 31u;
            const uint32_t bits = (mw >> sh) & ((1u << VEC) - 1u);
            uint32_t pos = run + me + __popc(mw & ((1u << sh) - 1u));
            union {
                uint4 v;
                T e[VEC];
            } x;
            x.v = lds128(seg + pass * WPP * 32 + g * 32 * VEC + lane * VEC);
#pragma unroll
            for (uint32_t e = 0; e < VEC; ++e) {
                if ((bits >> e) & 1u) stage[pos] = x.e[e];
                pos += (bits >> e) & 1u;
            }
        }
        run += pass_total;
    }
    return run;
}

template <typename T, int MODE, int S, int NC, int UT>
__global__ void __launch_bounds__(Roles<MODE>::NTHREADS, 1) k_compact_tma(const CompactParams p)
{
    constexpr int MSLOTS = Roles<MODE>::MSLOTS;
    using L = Layout<T, S, NC, MSLOTS, UT>;
    constexpr uint32_t U = L::U;
    constexpr uint32_t TE = L::TE;
    constexpr uint32_t W = L::W;
    constexpr uint64_t UE = static_cast<uint64_t>(U) * TE; // unit elements
    constexpr uint32_t VEC = 16 / sizeof(T);               // elements per 16-byte vector
    constexpr uint32_t E = TE / NC;                        // elements per compute warp
    constexpr uint32_t SW = E / 32;                        // mask words per compute warp
    constexpr uint32_t WPP = SW < 32 ? SW : 32;            // words per pass
    constexpr uint32_t PASSES = SW / WPP;
    constexpr uint32_t LPW_SCAN = 32 / NC;                 // scanner lanes per compute warp
    constexpr uint32_t KWORDS = W / 32;                    // mask words per lane per tile
    constexpr uint32_t SEG_COPY = TILE_BYTES / 32;         // producer skip granularity (bytes)
    static_assert(SW % WPP == 0 && WPP % VEC == 0, "pass/group shape");
    static_assert(LPW_SCAN >= 1, "at most 32 compute warps");

    extern __shared__ __align__(128) uint8_t smem[];
    __shared__ uint32_t s_flag;
    uint8_t* pay = smem + L::PAY;
    uint32_t* msk = reinterpret_cast<uint32_t*>(smem + L::MASK);
    uint8_t* outb = smem + L::OUTB;
    UnitMeta<U, NC>* meta = reinterpret_cast<UnitMeta<U, NC>*>(smem + L::META);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::BARS);
    uint64_t* full_pay = bars;                 // [S]  payload tile landed
    uint64_t* empty_pay = bars + S;            // [S]  payload tile consumed by all compute warps
    uint64_t* mask_full = bars + 2 * S;        // [MS] unit mask landed
    uint64_t* mask_empty = mask_full + MSLOTS; // [MS] unit finished by all compute warps
    uint64_t* ready = mask_empty + MSLOTS;     // [MS] unit offsets published by the scanner
    uint64_t* counted = ready + MSLOTS;        // [MS] 1-pass: unit counted, aggregate published

    const uint32_t warp = threadIdx.x >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    // the column of a unit of this launch, and the column named in a unit's meta
    auto col_of_unit = [&](uint64_t u) -> const ColumnDesc& { return column_of(p.col0, p.cols, p.unit_col, u); };
    auto col_at = [&](uint32_t c) -> const ColumnDesc& { return p.cols ? p.cols[c] : p.col0; };

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full_pay[s], 1);
            mbar_init(&empty_pay[s], NC); // one arrival per compute warp
        }
        for (int m = 0; m < MSLOTS; ++m) {
            mbar_init(&mask_full[m], 1);
            mbar_init(&mask_empty[m], NC);
            mbar_init(&ready[m], 1);
            mbar_init(&counted[m], 1);
        }
        fence_mbar_init();
    }
    __shared__ uint32_t s_hflags;
    grid_dependency_wait(); // everything below may read what earlier kernels wrote
    const uint32_t hflags = (MODE == 1) ? cta_header_flags(p.hdr, &s_hflags) : 3u; // also the init barrier
    if (MODE == 0) __syncthreads();
    const uint32_t epoch = (MODE == 0) ? p.hdr->epoch : 0u;
    const bool scan_ok = (hflags & 1u) != 0u; // 3-pass: pass 2 completed cleanly
    // 3-pass hybrid: some units may belong to the sparse gather kernel
    const bool hybrid = MODE == 1 && p.sparse_max != 0 && scan_ok && (hflags & 2u) != 0u;

    if (warp == 0) {
        // ------------------------------------------------------------- producer
        const uint64_t policy = l2_policy_evict_first();
        bool failed = false;
        // take the next unit id (warp-uniform)
        // 3-pass hybrid: window of 32 candidates from this CTA's round-robin unit list; bit k
        // of cand_bits set = candidate cand_base + k is a unit this kernel must process
        uint64_t cand_base = 0;
        uint32_t cand_bits = 0;
        bool cand_loaded = false;
        // 1-pass: lane 0 requests the NEXT ticket right after using the current one, so the
        // atomic's round trip overlaps a unit of streaming. A CTA's tickets still increase,
        // and the one left over at the end lies past the last unit, so no unit is dropped.
        uint32_t ticket_next = 0;
        bool ticket_pending = false;
        auto take_unit = [&](uint32_t j) -> uint64_t {
            if constexpr (MODE == 0) {
                uint32_t t = 0;
                if (lane == 0) {
                    t = ticket_pending ? ticket_next : atomicAdd(&p.hdr->tile_counter, 1u);
                    ticket_next = atomicAdd(&p.hdr->tile_counter, 1u);
                }
                ticket_pending = true;
                return __shfl_sync(0xffffffffu, t, 0);
            } else {
            if (!hybrid) return static_cast<uint64_t>(blockIdx.x) + static_cast<uint64_t>(j) * gridDim.x;
            while (cand_bits == 0u) {
                if (cand_loaded) cand_base += 32;
                cand_loaded = true;
                const uint64_t u = static_cast<uint64_t>(blockIdx.x) + (cand_base + lane) * gridDim.x;
                bool take = u >= p.num_tiles; // past the end: sentinel
                if (!take) {
                    const ColumnDesc& C = col_of_unit(u);
                    const uint64_t ul = u - C.unit_base;
                    const uint64_t e_b = ul * UE, e_e = (ul + 1) * UE;
                    const uint64_t off_b = chunk_offset(C, e_b >> p.chunk_log2, p.chunk_log2);
                    const uint64_t off_e =
                        e_e >= C.n ? *C.d_count : chunk_offset(C, e_e >> p.chunk_log2, p.chunk_log2);
                    take = off_e - off_b > p.sparse_max;
                }
                cand_bits = __ballot_sync(0xffffffffu, take);
            }
            const uint32_t k = __ffs(cand_bits) - 1;
            cand_bits &= cand_bits - 1;
            const uint64_t pick = static_cast<uint64_t>(blockIdx.x) + (cand_base + k) * gridDim.x;
            return pick < p.num_tiles ? pick : p.num_tiles;
            }
        };
        // arm mask slot j % MSLOTS with unit `unit` (or the end-of-work sentinel)
        auto issue_mask = [&](uint32_t j, uint64_t unit) -> bool {
            const uint32_t slot = j % MSLOTS;
            if (j >= (uint32_t)MSLOTS &&
                !mbar_wait_warp(&mask_empty[slot], ((j / MSLOTS) - 1) & 1u, p.timeout_ns, lane)) {
                if (lane == 0) record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                return false;
            }
            if (unit >= p.num_tiles) { // num_tiles holds the unit count
                if (lane == 0) {
                    meta[slot].unit = -1;
                    mbar_arrive(&mask_full[slot]);
                }
                return true;
            }
            uint32_t* dst = msk + slot * (U * W);
            const ColumnDesc& C = col_of_unit(unit);
            const uint64_t ul = unit - C.unit_base;
            if (lane == 0) {
                meta[slot].unit = static_cast<int64_t>(unit);
                meta[slot].ul = ul;
                meta[slot].col = p.cols ? __ldg(p.unit_col + unit) : 0u;
            }
            if ((ul + 1) * UE <= C.n) {
                if (lane == 0) {
                    mbar_arrive_expect_tx(&mask_full[slot], L::UMASK_BYTES);
                    bulk_g2s(dst, C.mask + ul * (U * W), L::UMASK_BYTES, &mask_full[slot]);
                }
            } else {
                // ragged last unit of the column: one bulk copy of the whole 16-byte groups of
                // complete words, plain loads for the rest (at most three complete words and
                // the partial last word), zeros past n. (A plain load per word made every
                // column's last unit cost its producer dozens of dependent loads.)
                const uint64_t w0 = ul * (U * W);
                const uint64_t full_col = C.n / 32; // complete words of the column
                const uint32_t full = full_col > w0 ? static_cast<uint32_t>(full_col - w0) : 0u; // < U * W
                const uint32_t bulk = full & ~3u;
                const uint32_t nval = static_cast<uint32_t>((C.n + 31) / 32 - w0); // words holding elements
                for (uint32_t i = bulk + lane; i < U * W; i += 32) {
                    uint32_t m = 0;
                    if (i < nval) {
                        m = __ldg(C.mask + w0 + i);
                        if (i == nval - 1 && (C.n & 31u)) m &= (1u << (C.n & 31u)) - 1u;
                    }
                    dst[i] = m;
                }
                __syncwarp();
                if (lane == 0) {
                    __threadfence_block();
                    if (bulk) {
                        mbar_arrive_expect_tx(&mask_full[slot], bulk * 4u);
                        bulk_g2s(dst, C.mask + w0, bulk * 4u, &mask_full[slot]);
                    } else {
                        mbar_arrive(&mask_full[slot]);
                    }
                }
            }
            return true;
        };

        uint32_t tseq = 0;        // payload stages armed so far
        uint32_t masks_armed = 0; // unit masks (or the end sentinel) armed so far
        bool ended = false;       // the end sentinel has been armed
        constexpr uint32_t AHEAD = Roles<MODE>::AHEAD;
        auto arm = [&](uint32_t jj) -> bool {
            const uint64_t u = take_unit(jj);
            if (!issue_mask(jj, u)) return false;
            ++masks_armed;
            ended = u >= p.num_tiles;
            return true;
        };
        for (uint32_t a = 0; a < AHEAD && !failed && !ended; ++a) failed = !arm(a);
        for (uint32_t j = 0; !failed; ++j) { // j: unit index of this CTA
            const uint32_t slot = j % MSLOTS;
            __syncwarp(); // lane 0's meta writes of the arming are visible to the warp
            if (meta[slot].unit < 0) break;
            const uint64_t cur = static_cast<uint64_t>(meta[slot].unit);
            if (!ended && !arm(j + AHEAD)) {
                failed = true;
                break;
            }
            const ColumnDesc& C = col_of_unit(cur);
            const uint64_t cul = cur - C.unit_base;
            const uint64_t rem_unit = C.n - cul * UE;
            const uint32_t ntiles = rem_unit >= UE ? U : static_cast<uint32_t>((rem_unit + TE - 1) / TE);
            // the unit's mask must have landed before segments can be skipped
            const bool use_skip = p.skip != 0u;
            if (use_skip && !mbar_wait_warp(&mask_full[slot], (j / MSLOTS) & 1u, p.timeout_ns, lane)) {
                if (lane == 0) record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                failed = true;
                break;
            }
            for (uint32_t k = 0; k < ntiles; ++k, ++tseq) {
                const uint32_t s = tseq % S;
                const uint32_t u = tseq / S;
                if (u > 0 && !mbar_wait_warp(&empty_pay[s], (u - 1) & 1u, p.timeout_ns, lane)) {
                    if (lane == 0) record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                    failed = true;
                    break;
                }
                const uint64_t tile = cul * U + k; // tile within the column
                const uint64_t rem = C.n - tile * TE;
                uint8_t* dst = pay + s * TILE_BYTES;
                const uint8_t* src = C.in + tile * TILE_BYTES;
                if (rem >= TE) {
                    // Choose how to fill the stage from the tile's landed mask:
                    //   none    : no selected element
                    //   runs    : >= 8 of 32 1 KB segments empty — one bulk copy per run of
                    //             non-empty segments
                    //   dense   : one bulk copy of the tile
                    // (A gather of only the 16-byte blocks holding selected elements, one
                    // cp.async each, was slower than these copies even at 8 selected per
                    // tile: the single producer warp issuing them became the bottleneck.)
                    uint32_t nz = 0xffffffffu;
                    const uint32_t* mw = msk + slot * (U * W) + k * W + lane * KWORDS;
                    if (use_skip) {
                        uint32_t any = 0;
#pragma unroll
                        for (uint32_t i = 0; i < KWORDS / 4; ++i) {
                            const uint4 q = lds128(mw + ((i + lane) % (KWORDS / 4)) * 4); // see MASK_ROT
                            any |= q.x | q.y | q.z | q.w;
                        }
                        nz = __ballot_sync(0xffffffffu, any != 0u);
                    }
                    if (nz == 0u) {
                        if (lane == 0) mbar_arrive(&full_pay[s]);
                    } else if (__popc(nz) <= 24) {
                        // runs of non-empty 1 KB segments, one bulk copy each
                        if (lane == 0) mbar_arrive_expect_tx(&full_pay[s], __popc(nz) * SEG_COPY);
                        __syncwarp();
                        const uint32_t starts = nz & ~(nz << 1);
                        if ((starts >> lane) & 1u) {
                            const uint32_t len = __clz(__brev(~(nz >> lane))); // consecutive non-empty segments
                            bulk_g2s_hint(dst + lane * SEG_COPY, src + lane * SEG_COPY, len * SEG_COPY, &full_pay[s],
                                          policy);
                        }
                    } else {
                        if (lane == 0) {
                            mbar_arrive_expect_tx(&full_pay[s], TILE_BYTES);
                            bulk_g2s_hint(dst, src, TILE_BYTES, &full_pay[s], policy);
                        }
                    }
                } else {
                    // ragged last tile: bulk copy of the 16-byte-multiple part, bytes for the rest
                    const uint32_t bytes = static_cast<uint32_t>(rem) * static_cast<uint32_t>(sizeof(T));
                    const uint32_t aligned = bytes & ~15u;
                    for (uint32_t b = aligned + lane; b < bytes; b += 32) dst[b] = __ldg(src + b);
                    __syncwarp();
                    if (lane == 0) {
                        __threadfence_block();
                        if (aligned) {
                            mbar_arrive_expect_tx(&full_pay[s], aligned);
                            bulk_g2s_hint(dst, src, aligned, &full_pay[s], policy);
                        } else {
                            mbar_arrive(&full_pay[s]);
                        }
                    }
                }
            }
            if (failed) break;
        }
        // Drain: the most recent arming of every payload stage and mask slot must have
        // landed before the CTA may exit (already true on the normal path).
        for (uint32_t k = 0; k < (uint32_t)S && k < tseq; ++k) {
            const uint32_t q = tseq - 1 - k;
            mbar_wait_warp(&full_pay[q % S], (q / S) & 1u, p.timeout_ns, lane);
        }
        for (uint32_t k = 0; k < (uint32_t)MSLOTS && k < masks_armed; ++k) {
            const uint32_t q = masks_armed - 1 - k;
            mbar_wait_warp(&mask_full[q % MSLOTS], (q / MSLOTS) & 1u, p.timeout_ns, lane);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------- scanner
        for (uint32_t j = 0;; ++j) {
            const uint32_t slot = j % MSLOTS;
            if (!mbar_wait_warp(&mask_full[slot], (j / MSLOTS) & 1u, p.timeout_ns, lane)) {
                if (lane == 0) record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                break;
            }
            const int64_t unit = meta[slot].unit;
            if (unit < 0) {
                if (lane == 0) mbar_arrive(MODE == 0 ? &counted[slot] : &ready[slot]);
                break;
            }
            const ColumnDesc& C = col_at(meta[slot].col);
            const uint64_t ul = meta[slot].ul;
            // in the 3-pass form start the offset load first; its latency hides under the popcounts
            uint64_t prefix = POISON;
            if (MODE == 1 && scan_ok) prefix = chunk_offset(C, (ul * UE) >> p.chunk_log2, p.chunk_log2);
            uint32_t unit_total = 0;
#pragma unroll
            for (uint32_t k = 0; k < U; ++k) {
                const uint32_t* mw = msk + slot * (U * W) + k * W + lane * KWORDS;
                uint32_t c = 0;
#pragma unroll
                for (uint32_t i = 0; i < KWORDS / 4; ++i) {
                    const uint4 q = lds128(mw + ((i + lane) % (KWORDS / 4)) * 4); // rotated: see MASK_ROT
                    c += __popc(q.x) + __popc(q.y) + __popc(q.z) + __popc(q.w);
                }
                const uint32_t incl = warp_incl_scan(c, lane);
                if ((lane % LPW_SCAN) == 0) meta[slot].warp_base[k][lane / LPW_SCAN] = unit_total + incl - c;
                unit_total += __shfl_sync(0xffffffffu, incl, 31);
            }
            if constexpr (MODE == 0) {
                // publish the aggregate now; the look-back warp resolves the prefix (statuses
                // of a column are indexed from its first unit)
                if (lane == 0) {
                    meta[slot].total = unit_total;
                    publish_aggregate(p.status + C.unit_base, ul, unit_total, epoch);
                }
                __syncwarp(); // orders every lane's meta writes before lane 0's release
                if (lane == 0) mbar_arrive(&counted[slot]);
                continue;
            }
            if (prefix != POISON && prefix + unit_total > C.n) {
                if (lane == 0) record_error(p.hdr, DEVERR_RANGE);
                prefix = POISON;
            }
            if (lane == 0) meta[slot].prefix = prefix;
            __syncwarp(); // orders every lane's meta writes before lane 0's release
            if (lane == 0) mbar_arrive(&ready[slot]);
        }
    } else if (static_cast<int>(warp) == Roles<MODE>::LOOKBACK) {
        // ------------------------------------------------------------- look-back (1-pass)
        for (uint32_t j = 0;; ++j) {
            const uint32_t slot = j % MSLOTS;
            if (!mbar_wait_warp(&counted[slot], (j / MSLOTS) & 1u, p.timeout_ns, lane)) {
                if (lane == 0) record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                break;
            }
            const int64_t unit = meta[slot].unit;
            if (unit < 0) {
                if (lane == 0) mbar_arrive(&ready[slot]);
                break;
            }
            const ColumnDesc& C = col_at(meta[slot].col);
            const uint64_t ul = meta[slot].ul;
            const uint32_t unit_total = meta[slot].total;
            uint64_t prefix = lookback_warp<1, true>(p.status + C.unit_base, ul, unit_total, epoch, p.timeout_ns,
                                                     p.hdr, lane);
            if (prefix != POISON && prefix + unit_total > C.n) {
                if (lane == 0) record_error(p.hdr, DEVERR_RANGE);
                prefix = POISON;
            }
            if (lane == 0) {
                meta[slot].prefix = prefix;
                if (ul == (C.n + UE - 1) / UE - 1) // the column's last unit
                    *C.d_count = (prefix == POISON) ? POISON : prefix + unit_total;
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&ready[slot]);
        }
    } else {
        // ------------------------------------------------------------- compute
        const uint32_t cw = warp - Roles<MODE>::FIRST_COMPUTE;
        T* stage = reinterpret_cast<T*>(outb + cw * L::STAGE_OUT_BYTES);
        uint32_t tseq = 0;
        bool failed = false;
        for (uint32_t j = 0; !failed; ++j) {
            const uint32_t slot = j % MSLOTS;
            if (!mbar_wait_warp(&ready[slot], (j / MSLOTS) & 1u, p.timeout_ns, lane)) {
                if (lane == 0) record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                break;
            }
            const int64_t unit = meta[slot].unit;
            if (unit < 0) break;
            const uint64_t prefix = meta[slot].prefix;
            const bool write = prefix != POISON;
            const ColumnDesc& C = col_at(meta[slot].col);
            uint8_t* const col_out = C.out;
            const uint64_t rem_unit = C.n - meta[slot].ul * UE;
            const uint32_t ntiles = rem_unit >= UE ? U : static_cast<uint32_t>((rem_unit + TE - 1) / TE);
            for (uint32_t k = 0; k < ntiles; ++k, ++tseq) {
                const uint32_t s = tseq % S;
                if (!mbar_wait_warp(&full_pay[s], (tseq / S) & 1u, p.timeout_ns, lane)) {
                    if (lane == 0) record_error(p.hdr, DEVERR_PIPELINE_TIMEOUT);
                    failed = true;
                    break;
                }
                const uint64_t gpos = prefix + meta[slot].warp_base[k][cw];
                const uint32_t a = static_cast<uint32_t>(gpos % VEC);
                uint32_t run = a;
                if (write) {
                    const T* seg = reinterpret_cast<const T*>(pay + s * TILE_BYTES) + cw * E;
                    const uint32_t* segm = msk + slot * (U * W) + k * W + cw * SW;
                    // 1- and 2-byte elements, and the 1-pass form: loads and shuffles first
                    if constexpr (sizeof(T) <= 2 || MODE == 0)
                        run = place_vectors<T, PASSES, WPP>(seg, segm, stage, run, lane);
                    else
                        run = place_grouped<T, PASSES, WPP>(seg, segm, stage, run, lane);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&empty_pay[s]); // this warp no longer reads payload stage s
                if (write) {
                    const uint32_t nvec = (run + VEC - 1) / VEC;
                    uint8_t* gdst = col_out + (gpos - a) * sizeof(T);
                    for (uint32_t v = lane; v < nvec; v += 32) {
                        const uint32_t e0 = v * VEC;
                        const uint32_t e1 = e0 + VEC;
                        if (e0 >= a && e1 <= run) {
                            stg128_cs(gdst + v * 16u, lds128(stage + e0));
                        } else {
                            const uint32_t lo = e0 > a ? e0 : a;
                            const uint32_t hi = e1 < run ? e1 : run;
                            for (uint32_t e = lo; e < hi; ++e) reinterpret_cast<T*>(gdst)[e] = stage[e];
                        }
                    }
                }
                __syncwarp();
            }
            if (failed) break;
            __syncwarp();
            if (lane == 0) mbar_arrive(&mask_empty[slot]); // this warp no longer reads the unit's mask/meta
        }
    }

    if (MODE == 0)
        lookback_kernel_epilogue(p.hdr, &p.hdr->tile_counter, &p.hdr->done_counter, &s_flag, false, p.keep_begin,
                                 p.keep_end);
}

// ---------------------------------------------------------------------------------
// Host side: per-device attribute setup and dispatch. Variants: 0 = 1-pass with units of
// UNIT_TILES tiles, 1 = 3-pass writeout (UNIT_TILES), 2 = 1-pass with one-tile units (short
// columns: four times as many units, so more SMs take part), 3 = 1-pass with a deeper payload
// ring for long columns of 4- and 8-byte elements (mode 2; the same kernel as 0 otherwise).
// ---------------------------------------------------------------------------------
namespace {
constexpr int MAX_DEVICES = 64;
constexpr int VARIANTS = 4;
// bit (wi * VARIANTS + variant) set once the smem attribute was applied on that device
unsigned g_attr_done[MAX_DEVICES];

template <int V>
struct Variant {
    static constexpr int MODE = V == 1 ? 1 : 0;
    static constexpr int UT = V == 2 ? 1 : static_cast<int>(UNIT_TILES);
    static constexpr bool DEEP = V == 3;
};

template <typename T, int V>
struct Kernel {
    static constexpr int MODE = Variant<V>::MODE;
    // Payload stages: one more for long 1-pass columns of 4- and 8-byte elements, whose reads
    // then have 160 KB in flight per SM (measured +1.9 to +2.7% at 2^28; slower at 2^24 and
    // in the 3-pass writeout, and the 1- and 2-byte layouts have no room).
    static constexpr int S = (Variant<V>::DEEP && sizeof(T) >= 4) ? STAGES + 1 : STAGES;
    using L = Layout<T, S, NCW, Roles<MODE>::MSLOTS, Variant<V>::UT>;
    static constexpr uint32_t SMEM = L::TOTAL;
    static constexpr uint32_t THREADS = Roles<MODE>::NTHREADS;
    static void (*fn())(CompactParams) { return k_compact_tma<T, MODE, S, NCW, Variant<V>::UT>; }
};

template <typename T, int V>
cudaError_t ensure_attr(int dev)
{
    constexpr int wi = (sizeof(T) == 1) ? 0 : (sizeof(T) == 2) ? 1 : (sizeof(T) == 4) ? 2 : 3;
    const unsigned bit = 1u << (wi * VARIANTS + V);
    if (dev >= 0 && dev < MAX_DEVICES && (__atomic_load_n(&g_attr_done[dev], __ATOMIC_ACQUIRE) & bit)) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(Kernel<T, V>::fn(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(Kernel<T, V>::SMEM));
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < MAX_DEVICES) __atomic_fetch_or(&g_attr_done[dev], bit, __ATOMIC_RELEASE);
    return cudaSuccess;
}

template <typename T, int V>
cudaError_t launch_t(const CompactParams& p, uint32_t grid, cudaStream_t stream)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    e = ensure_attr<T, V>(dev);
    if (e != cudaSuccess) return e;
    e = launch_pdl(Kernel<T, V>::fn(), dim3(grid), dim3(Kernel<T, V>::THREADS), Kernel<T, V>::SMEM, stream, p);
    note_launch();
    return e;
}

template <typename T, int V>
int blocks_per_sm_t()
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (ensure_attr<T, V>(dev) != cudaSuccess) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, Kernel<T, V>::fn(), Kernel<T, V>::THREADS,
                                                      Kernel<T, V>::SMEM) != cudaSuccess)
        return 0;
    return nb;
}

int variant_of(int mode, uint32_t unit_tiles)
{
    if (mode == 1) return unit_tiles == UNIT_TILES ? 1 : -1;
    if (mode == 0) return unit_tiles == UNIT_TILES ? 0 : unit_tiles == 1 ? 2 : -1;
    if (mode == 2) return unit_tiles == UNIT_TILES ? 3 : -1;
    return -1;
}

// the deep variant exists for 4- and 8-byte elements only; narrower ones run variant 0
template <typename T>
int variant_for(int v)
{
    return (v == 3 && sizeof(T) < 4) ? 0 : v;
}

template <typename T>
uint32_t smem_t(int v)
{
    v = variant_for<T>(v);
    if constexpr (sizeof(T) >= 4)
        if (v == 3) return Kernel<T, 3>::SMEM;
    return v == 0 ? Kernel<T, 0>::SMEM : v == 1 ? Kernel<T, 1>::SMEM : Kernel<T, 2>::SMEM;
}

template <typename T>
int blocks_t(int v)
{
    v = variant_for<T>(v);
    if constexpr (sizeof(T) >= 4)
        if (v == 3) return blocks_per_sm_t<T, 3>();
    return v == 0 ? blocks_per_sm_t<T, 0>() : v == 1 ? blocks_per_sm_t<T, 1>() : blocks_per_sm_t<T, 2>();
}

template <typename T>
cudaError_t launch_v(int v, const CompactParams& p, uint32_t grid, cudaStream_t stream)
{
    v = variant_for<T>(v);
    if constexpr (sizeof(T) >= 4)
        if (v == 3) return launch_t<T, 3>(p, grid, stream);
    return v == 0 ? launch_t<T, 0>(p, grid, stream) : v == 1 ? launch_t<T, 1>(p, grid, stream)
                                                             : launch_t<T, 2>(p, grid, stream);
}
} // namespace

uint32_t compact_tma_smem_bytes(uint32_t elem_bytes, int mode, uint32_t unit_tiles)
{
    const int v = variant_of(mode, unit_tiles);
    if (v < 0) return 0;
    switch (elem_bytes) {
        case 1: return smem_t<uint8_t>(v);
        case 2: return smem_t<uint16_t>(v);
        case 4: return smem_t<uint32_t>(v);
        case 8: return smem_t<uint64_t>(v);
        default: return 0;
    }
}

int compact_tma_blocks_per_sm(uint32_t elem_bytes, int mode, uint32_t unit_tiles)
{
    const int v = variant_of(mode, unit_tiles);
    if (v < 0) return 0;
    switch (elem_bytes) {
        case 1: return blocks_t<uint8_t>(v);
        case 2: return blocks_t<uint16_t>(v);
        case 4: return blocks_t<uint32_t>(v);
        case 8: return blocks_t<uint64_t>(v);
        default: return 0;
    }
}

cudaError_t launch_compact_tma(const CompactParams& p, uint32_t elem_bytes, int mode, uint32_t grid, cudaStream_t stream,
                               uint32_t unit_tiles)
{
    const int v = variant_of(mode, unit_tiles);
    if (v < 0) return cudaErrorInvalidValue;
    switch (elem_bytes) {
        case 1: return launch_v<uint8_t>(v, p, grid, stream);
        case 2: return launch_v<uint16_t>(v, p, grid, stream);
        case 4: return launch_v<uint32_t>(v, p, grid, stream);
        case 8: return launch_v<uint64_t>(v, p, grid, stream);
        default: return cudaErrorInvalidValue;
    }
}

} // namespace cs
