// Kernel launchers of the B200 trace (defined in st_kernels_fp64.cu,
// st_kernels_mixed.cu and st_kernels_common.cu).
#pragma once
#include <cuda_runtime.h>
#include <cstdint>
#include "st_scene.h"

namespace stb {

constexpr int kProbeBlock = 256;
constexpr int kResolveBlock = 128;  // threads per block of the grid probe's element-test kernel
constexpr int kCandPerThread = 8;   // sun rays per thread of the grid probe's pre-test kernel
constexpr int kCandRays = kProbeBlock * kCandPerThread;
constexpr int kTraceBlock = 128;
// register-budget variants of the probe and trace kernels (minimum resident blocks per
// SM given to __launch_bounds__); all compute the same results
constexpr int kProbeVariants = 3;
constexpr int kProbeMinBlocks[kProbeVariants] = {4, 6, 8};
// resident blocks per SM asked of the trace's shade and search kernels (register budget)
constexpr int kWfShadeMinBlocks = 4;
constexpr int kWfSearchMinBlocks = 4;
// Search kinds: the trace's search kernel is compiled once per kind, holding only the code
// its stages need (fewer registers, more resident warps).  Bits: kSearchFlat, the stage holds
// flat elements only; kSearchBrute, the stage has neither ground grid nor BVH (few elements,
// tested one after the other); kSearchClosed, the stage's surfaces are all closed-form (set
// only without kSearchFlat, which implies it).
constexpr int kSearchFlat = 1, kSearchBrute = 2, kSearchClosed = 4, kSearchKinds = 8;
__host__ __device__ inline int stage_search_kind(const StageRec &st) {
    return (st.flat_only ? kSearchFlat : (st.closed_only ? kSearchClosed : 0)) |
           ((!st.grid_on && st.bvh_off < 0) ? kSearchBrute : 0);
}
constexpr int kWfBruteMinBlocks = 8;      // search kernels of stages tested element by element
constexpr int kWfFlatSearchMinBlocks = 5;  // search kernels of flat-only stages
constexpr int kWfFirstFlatMinBlocks = 8;   // first kernel on a flat-only first stage (FP64)
#ifndef ST_FIRST_FLAT_MINB_MIXED
#define ST_FIRST_FLAT_MINB_MIXED 8
#endif
constexpr int kWfFirstFlatMinBlocksMixed = ST_FIRST_FLAT_MINB_MIXED;  // the same in mixed precision

// shade kernel of scenes with closed-form surfaces only: FP64 (5 blocks per SM measured faster
// than 4 and no slower than 6) and mixed precision (4; 5 and 6 no faster)
constexpr int kWfClosedShadeMinBlocks = 5;
constexpr int kWfClosedShadeMinBlocksMixed = 4;
#ifndef ST_EXACT_PROBE_MINB
#define ST_EXACT_PROBE_MINB 8
#endif
constexpr int kExactProbeMinBlocks = ST_EXACT_PROBE_MINB;  // mixed probe of flat rectangles (k_sun_probe_exact)

enum RunFlags : unsigned {
    kFlagHitCap = 1u,         // a ray reached kMaxHitsPerStage in one stage
    kFlagBadInteraction = 2u, // interaction type other than 1 or 2 (raytrace.cpp:943-946)
    kFlagRecordOverflow = 4u,
};

struct RunCounters {
    unsigned long long stage_entries[kMaxStages];
    unsigned int max_enter[kMaxStages];   // largest ray number entering stage i
    unsigned int max_ttmiss[kMaxStages];  // largest ray number missing trace-through stage i
    unsigned long long records;
    unsigned int flags;
    unsigned int pad_;
};

// Device-side progress of a run: the ray-number cut-off at the requested hit
// count is applied on the device, so batches can be queued without host syncs.
struct RunState {
    unsigned long long hits_done;  // rays numbered so far
    unsigned long long target;     // rays to number (~0 in explicit-ray mode)
    unsigned long long sun_rays;   // SunRayCount so far (final once reached)
    unsigned int reached;
    unsigned int cursor;           // trace work queue: next hit-list entry to hand out
    unsigned long long cut_sid;    // sun-ray index of the batch's last numbered hit (set by the sort)
};

// Per-ray state of the trace between its kernels, one slot per hit-list entry of a batch
// (structure of arrays; component q of a vector at [q * cap + slot]).
struct WfState {
    uint64_t *sid;      // sun-ray index (random stream key)
    uint32_t *raynum;
    uint32_t *draw;     // next draw of the ray's random stream
    int4 *meta;         // stage, hits in the stage, element left (flat, else -1), element to shade (-1)
    int *fe0;           // the ray's first first-stage element (global index), -1 none
    double *p, *c;      // position, direction: global while the stage has no hit yet, else stage frame
    uint32_t cap;
};

// Queues of the trace.  Search queues come per search kind present in the scene (the
// kernel variant that searches the rays' stages) and per round parity; one shade queue.
// Queue k of parity p holds up to `cap` entries at search[p] + k * cap.  Counts, per
// round r at r * (n_queues + 1): the n_queues search counts, then the shade count; the
// finishing kernel takes the search counts of round `rounds`.  The launcher zeroes them.
struct WfQueues {
    uint32_t *search[2];
    uint32_t *shade;
    uint32_t *counts;                     // (rounds + 1) * (n_queues + 1) entries
    uint32_t cap;
    int rounds;
    int n_queues;
    int queue_kind[kMaxStages];           // search kind of queue k
    unsigned char stage_queue[kMaxStages];  // search queue of the rays of stage s
};

struct TraceOut {
    RecordDev *recs;
    unsigned long long rec_cap;
    unsigned long long *rec_count;   // records written by this batch (slots beyond rec_cap dropped)
    RunCounters *ctr;
    unsigned long long *first_hits;  // per global element index
    unsigned long long *absorbed;
    unsigned long long *delivered;   // per global element index (first-stage elements)
    // stage-data saving (st_b200_set_save_stage_data): rays leaving stage 1 and stage 2
    // (global position, direction, ray number: 7 doubles per row), null when off
    double *save_rows[2];
    unsigned long long *save_count[2];
    unsigned long long save_cap;
};

// Rays entering the second stage from saved stage data (replay, st_b200_sim_run_replay):
// 7 doubles per row (global position, direction, ray number) and the global index of each
// ray's first first-stage element (-1 unknown).
struct ReplayIn {
    const double *rows;
    const int *fe0;
    uint32_t n;
};


// Outputs of the first-stage probe of sun rays [s0, s0 + n):
//   block_counts  hits of every kProbeBlock rays (always written);
//   hit_elem      optional: element + 1 or 0 per ray;
//   cand, cand_count  the probe's ray list (room for n entries) and its length: the grid
//                 probe's candidates, or (with cand_el) every ray of the other probes;
//   cand_el       optional: element + 1 or 0 per list entry;
//   hit_mask      optional: one bit per ray, set for a hit (hit_mask_words(n) words);
//   amb, amb_count  room for n ray indices and their count (k_sun_probe_exact only).
// One numbered hit of a batch, sorted by first-stage element: its sun-ray index, the element
// and its rank among the batch's hits in sun-ray order (its ray number less the batch's base);
// one 16-byte store per hit when the sort scatters it.
struct __align__(16) HitRec {
    unsigned long long sid;
    uint32_t el, rank;
};

struct ProbeOut {
    uint32_t *block_counts;
    uint32_t *hit_elem;
    uint32_t *cand, *cand_count, *cand_el;
    uint32_t *hit_mask;
    uint32_t *amb, *amb_count;  // mixed probe of flat rectangles: rays left to the double search
};
// hit-mask words for n sun rays, rounded up to whole blocks of the widest probe variant
// (16 rays per thread): every probe kernel writes the words of its blocks in full
constexpr int kMaskRays = kProbeBlock * 16;
constexpr size_t hit_mask_words(uint64_t n) { return size_t((n + kMaskRays - 1) / kMaskRays) * (kMaskRays / 32); }
// rays per thread of the mixed flat-rectangle probe, per autotuner variant
constexpr int kExactRpt[kProbeVariants] = {4, 8, 16};

// First-stage probe of sun rays [s0, s0 + n) into `o`.  Returns the number of kernels
// launched.
int launch_probe_fp64(const SceneDev &S, uint64_t s0, uint32_t n, const ProbeOut &o, const RunState *rs,
                      int variant, cudaStream_t st);
int launch_probe_mixed(const SceneDev &S, uint64_t s0, uint32_t n, const ProbeOut &o, const RunState *rs,
                       int variant, cudaStream_t st);
// first kernel of the grid probe (shared by both precisions)
void launch_sun_candidates(const SceneDev &S, uint64_t s0, uint32_t n, const ProbeOut &o, const RunState *rs,
                           cudaStream_t st);
// Trace of a batch's numbered rays (sorted hits whose rank lies below the cut-off at the
// requested hit count): the first kernel, `Q.rounds` rounds of search and shade kernels,
// and the finishing kernel.  Returns the number of kernels launched.
// With `replay` (non-null) the rays enter the second stage from saved rows instead of the
// hit list (hits and total are then unused).
int launch_trace_fp64(bool records, const SceneDev &S, const HitRec *hits, const uint32_t *total,
                      const RunState *rs, const TraceOut &O,
                      const WfState &W, const WfQueues &Q, const ReplayIn *replay, cudaStream_t st);
int launch_trace_mixed(bool records, const SceneDev &S, const HitRec *hits, const uint32_t *total,
                       const RunState *rs, const TraceOut &O,
                       const WfState &W, const WfQueues &Q, const ReplayIn *replay, cudaStream_t st);
// The batch's hits, from the probe's list (cand, cand_el, hit_mask) and the exclusive
// scan of its block counts (offsets, total), counting-sorted by first-stage element into
// `hits` (sun-ray index, element, rank of the hit in sun-ray order); the
// hit ranked last below the cut-off at the requested hit count leaves its sun-ray index in
// rs->cut_sid.  max_n bounds the list length (grid sizing).
void launch_list_sort(uint64_t s0, const ProbeOut &o, const uint32_t *offsets, const uint32_t *total, RunState *rs,
                      uint32_t n_elem0, uint32_t *elem_count, uint32_t *elem_cursor, uint32_t *scratch_total,
                      HitRec *hits, uint32_t max_n, cudaStream_t st);
// finite-element interpolation failures flagged by the kernels since the last call
unsigned take_fe_failures_fp64();
unsigned take_fe_failures_mixed();
void launch_offsets(const uint32_t *counts, uint32_t nb, uint32_t *offsets, uint32_t *total, cudaStream_t st);
// the same exclusive scan over the whole grid (two kernels); `parts` holds scan_parts(nb)
// chunk sums
void launch_scan(const uint32_t *counts, uint32_t nb, uint32_t *offsets, uint32_t *total, uint32_t *parts,
                 cudaStream_t st);
constexpr int kScanChunk = 2048, kScanBlock = 256;
constexpr size_t scan_parts(uint32_t nb) { return (size_t(nb) + kScanChunk - 1) / kScanChunk + 1; }
// the same scan for arrays of any length (up to 2^31 entries): chunk sums, their scan, and
// the chunks' scans from it.  offsets may be counts (in place).  parts holds
// scan_parts(nb) entries, parts2 scan_parts(scan_parts(nb)).
void launch_scan_large(const uint32_t *counts, uint32_t nb, uint32_t *offsets, uint32_t *total, uint32_t *parts,
                       uint32_t *parts2, cudaStream_t st);

// Ordering of a run's records on the device (the reference's readback order,
// TRayData::Merge in types.cpp:311-355): records are counted per (stage, ray number), the
// counts scanned into the first slot of every key, and each record is written to the slot
// of its key plus its hit index, mapped through the block-merge runs of its stage, as
// columns.
struct RecOrder {
    const RecordDev *recs;
    unsigned long long n;
    uint32_t rb;                     // ray numbers 0..rb per stage (key space nst * (rb + 1))
    int nst;
    int drop_later;                  // the records of every stage after the first are dropped
    uint32_t tt_drop[kMaxStages];    // per stage: the ray number whose miss record is dropped (0: none)
    uint32_t *key;                   // per key: count, then (after the scan) its first slot
    unsigned long long *stage_count; // kept records per stage
    const uint32_t *run_src, *run_dst;  // merge runs, stage by stage, by start in the stage's order
    const int *run_seg;              // the runs of stage s are [run_seg[s], run_seg[s + 1])
    double *col_d;                   // x, y, z, cx, cy, cz: 6 columns of `total` doubles
    int *col_i;                      // element, stage, ray number: 3 columns of `total` ints
    unsigned long long total;        // kept records
    unsigned int *bad;               // set when a record lies outside the key space
};
void launch_rec_count(const RecOrder &o, cudaStream_t st);
void launch_rec_scatter(const RecOrder &o, cudaStream_t st);
// batched runs with tracking: element e of `el` (n elements) takes the stage -> element
// rotation rot[9e .. 9e + 8]
void launch_set_rotations(ElemRec *el, uint32_t n, const double *rot, cudaStream_t st);

void launch_compact(uint64_t s0, uint32_t n, const uint32_t *hit_elem, const uint32_t *counts,
                    const uint32_t *offsets, uint64_t *hit_sid, uint32_t *hit_el, cudaStream_t st);
// cut-off and run state after a batch; the last numbered sun ray is read from the
// sun-ray-ordered hit list `hit_sid`, or from rs->cut_sid when it is null
void launch_advance(const uint32_t *total, const uint64_t *hit_sid, uint64_t s0, uint32_t n, RunState *rs,
                    cudaStream_t st);
}  // namespace stb
