// Label-propagation kernels: launch-argument structs and kernel declarations.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "common.cuh"

namespace lpa_dev {

// Kernel variants (all produce identical labels).
enum Variant : int {
  kVarWarp = 0,     // V1: lane-per-vertex decode, warp-per-vertex counting (deg <= kV1MaxDeg)
  kVarPacked = 1,   // V2: lane-per-vertex decode, several vertices per warp counting (deg <= 32)
  kVarBlock = 2,    // V3: block per vertex, segment-parallel decode, block table / sketch
  kVarTwoPass = 3,  // V4: a decode pass writes a CSR scratch; counting reads it
  kNumVariants = 4,
  kVarPackedLanes = 5  // batch plans only: V2 on a tiny segment, one thread per position (packed_vertex)
};

constexpr int kThreads = 256;             // threads per block of the iteration kernel
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kStage = 8192;         // staged ids/labels per block (1024 per warp)
constexpr uint32_t kTableSlots = 8192;    // 64-bit exact-count slots per block (1024 per warp)
constexpr uint32_t kWarpStage = kStage / kWarps;
constexpr uint32_t kWarpSlots = kTableSlots / kWarps;
constexpr uint32_t kV1MaxDeg = kWarpSlots - 1;         // 1023: a warp's table holds every distinct label
constexpr uint32_t kV2MaxDeg = 32;
constexpr uint32_t kBlockMaxSmemDeg = kTableSlots / 2; // exact degrees counted in shared memory (<= 4095)

// dynamic shared memory of the iteration kernel
constexpr size_t kSmemBytes = size_t(kStage) * 4 + size_t(kTableSlots) * 8;

struct Seg {
  uint32_t begin, end;  // positions [begin, end)
};

// A work item with the device range it will read, so a warp or block can
// prefetch items it has claimed but not started.
struct WorkItem {
  uint32_t tag;        // heavy: segment id; light: (segment << 3) | 32-position chunk
  uint32_t pf_bytes;   // bytes of the range to prefetch
  uint64_t pf_addr;    // device address of the range (bitstream bits, small-CSR ids or scratch ids)
};

// Work of the two-pass pre-pass: nlanes (<= 32) consecutive segments of the
// positions p0, p0 + 1, ..., starting at segment j0 of p0 (interval segments
// first, then residual ones) and spanning at most 32 positions.  seg is the
// plan segment its cycles are booked to.
struct DecodeGroup {
  uint32_t p0, j0, nlanes, seg;
  uint64_t w0;      // the stream words its segments read: [w0, w0 + wn)
  uint32_t wn, pad;
};
// staged ids per warp of the pre-pass: 1024 (32 KB per block with the lane in
// the ids' top bits) beat 768 by 1.5 %; 1280 and 1536 shrink L1 and lose 3 %
// and 13 % (R-MAT scale 24)
constexpr uint32_t kDecodeWindow = 1024;
// decode groups a warp of the pre-pass claims from its work queue at once
constexpr uint32_t kGroupClaim = 4;
// lpa_tune.gather_cache 0: the pre-pass reads the labels of ids below this
// through L1 (32 KB of labels), the others through L2 only
constexpr uint32_t kHotIds = 8192;
// lpa_tune.stage_stream 2: words of a group's stream span one shared-memory
// buffer holds (32 segments of < 512 bits plus their headers fit)
constexpr uint32_t kSpanWords = 576;
constexpr uint32_t kSpanSmemBytes = kWarps * 2 * kSpanWords * 4;  // its two buffers per warp (dynamic)

// Work of the two-pass count pass (k_count_two_pass): positions p0 ..
// p0 + np - 1, all of one kind, whose labels the pre-pass wrote to the
// scratch.  seg is the plan segment the cycles are booked to.
enum CountKind : uint32_t {
  kCountGroups = 0,  // np <= 32 positions of degree <= 32: G-lane groups, several vertices per round
  kCountWarp = 1,    // np <= 4 positions of degree <= kCountWarpMax: warp per vertex, 512-slot table
  kCountBlock = 2,   // one position, degree <= kCountBlockMax: block per vertex, 4096-slot table
  kCountSketch = 3,  // one position at or above the sketch threshold: block per vertex
};
struct CountItem {
  uint32_t p0, np, seg, kind;
};
// A block item of the count pass, with everything its block needs up front.
struct BlockItem {
  uint64_t ao;              // scratch index of the position's labels (arc offset)
  uint32_t p, d, node;      // position, degree, vertex id
  uint32_t seg, kind, pad;  // plan segment (cycles), kCountBlock or kCountSketch
};
constexpr uint32_t kCountWarpSlots = 512;
constexpr uint32_t kCountWarpMax = kCountWarpSlots - 1;  // tables fill up to load 1 (triangular probing)
constexpr uint32_t kCountBlockSlots = kWarps * kCountWarpSlots;  // the warps' tables together
// with lpa_tune.bulk_stage, group items of the count pass with at least this
// many scratch labels are staged by one bulk copy (cp.async.bulk) instead of
// per-lane loads
constexpr uint32_t kBulkMinLabels = 64;
constexpr uint32_t kBulkWaitTries = 1u << 22;  // mbarrier try_wait attempts before a copy counts as lost
constexpr uint32_t kCountBlockMax = 2047;
constexpr uint32_t kCountSmemBytes = kCountBlockSlots * 8;        // 32 KB

// Work of k_packed: up to 32 consecutive positions of one plan segment whose
// degrees are all <= kPackedMaxDeg, one lane each.
struct PackedChunk {
  uint32_t p0, np, seg, pad;
};
constexpr uint32_t kPackedMaxDeg = 15;  // the tiny bucket (degree < 16)

constexpr int kBusyKernels = 4;  // kernels of an iteration with a busy span (IterArgs::ktime)

// Work-queue counters of one iteration (IterArgs::work + kWorkCounters *
// slot): k_iterate's heavy items and light chunks, the count pass's block and
// warp items, the pre-pass's decode groups; the rest unused.
enum WorkCounter : int { kWqHeavy = 0, kWqLight, kWqBlock, kWqWarp, kWqGroups, kWorkCounters = 8 };

struct IterArgs {
  DevGraph g;
  uint32_t *labs0, *labs1;      // the two label buffers
  uint32_t parity0;             // iteration 0 of this launch reads labs0 when 0, labs1 when 1
  const uint32_t *it_dev;       // device iteration counter (CUDA-graph loop), nullptr: 0
  unsigned long long *changed;  // changed counters, indexed by the iteration counter
  uint32_t *work;               // work-queue counters: kWorkCounters per iteration slot
  uint32_t *err;
  const Seg *segs;              // all segments
  const uint8_t *seg_var;       // variant per segment
  const WorkItem *heavy;        // block work items (one segment each), largest first
  uint32_t n_heavy;
  const WorkItem *light;        // warp work items (32-position chunks)
  uint32_t n_light;
  const DecodeGroup *groups;    // two-pass pre-pass work: 32 segments per group
  uint32_t n_groups;
  const uint4 *pidx;            // per compressed position: {ibase - offset, rbase - offset, nseg_i, nseg_r}
  const BlockItem *cblock;      // count-pass block items (largest first)
  uint32_t n_cblock;
  const CountItem *cwarp;
  uint32_t n_cwarp;
  uint32_t warp_claim;          // warp items a warp of the count pass claims at once
  const PackedChunk *packed;    // k_packed work
  uint32_t n_packed;
  uint32_t cw_packed;           // cost weight of a k_packed warp-cycle (as cw_iterate)
  uint32_t *cursor;             // per compressed position: labels written by the pre-pass (pass 2 resets)
  long long *seg_cycles;        // per-segment device cycles (nullptr: off)
  // weights of one warp-cycle of k_iterate / k_decode_two_pass /
  // k_count_two_pass in seg_cycles: 960 / (the kernel's resident warps per
  // SM), so a booked unit is the same share of an SM whichever kernel spent it
  uint32_t cw_iterate, cw_decode, cw_count;
  // nullptr, or the busy span of each kernel of the iteration on the GPU's
  // clock (ns): ktime[k] = earliest warp start, ktime[kBusyKernels + k] =
  // latest warp end, k = 0 k_decode_two_pass, 1 k_count_two_pass, 2 k_iterate,
  // 3 k_packed
  unsigned long long *ktime;
  uint32_t *seg_changed;        // per-segment changed counts (nullptr: off)
  uint32_t cms_thr;             // 0: no sketch
  uint32_t seeds[kCmsDepth];
  // two-pass scratch: the neighbours of compressed position p at
  // scratch[arc_off[p]..), as labels in any order (k_decode_two_pass) or as
  // ids (scratch_labels == 0)
  uint32_t *scratch;
  const uint64_t *arc_off;
  uint32_t scratch_labels;      // 1: the scratch holds labels (the pre-pass), 0: ids
  // global exact-count tables for exact vertices above kBlockMaxSmemDeg
  uint32_t *gtab;
  uint32_t gtab_slots;          // slots per block (power of two), 0: none
  // graphs concatenated into one (a lockstep batch): graph k owns the vertex
  // ids [gbase[k], gbase[k + 1]); n_gbase = 0: one graph
  const uint32_t *gbase;
  uint32_t n_gbase;
  // stream words [0, wend) that bulk copies may read (a multiple of 4: the
  // copies move whole 16-byte units inside the stream's allocation)
  uint64_t wend;
  // per block of k_iterate: hub_spill_words labels of the sketch hub it is
  // decoding (nullptr: none; a hub decodes twice)
  uint32_t *hub_spill;
  uint32_t hub_spill_words;
};

// The id base of the graph that owns vertex `node`.  The sketch hashes a
// label relative to it, so a graph's sketch counts are those of the graph run
// alone; the exact paths compare labels only and need no base.
__device__ __forceinline__ uint32_t label_base(const IterArgs &a, uint32_t node) {
  if (a.n_gbase == 0) return 0u;
  uint32_t lo = 0, hi = a.n_gbase;  // gbase[lo] <= node < gbase[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(a.gbase + mid) <= node) lo = mid;
    else hi = mid;
  }
  return __ldg(a.gbase + lo);
}

__device__ __forceinline__ uint32_t iter_index(const IterArgs &a) { return a.it_dev ? *a.it_dev : 0u; }

// ---- many graphs in one persistent launch ------------------------------
struct BatchGraph {
  DevGraph g;
  uint32_t *labs0, *labs1;
  const Seg *segs;
  const uint8_t *seg_var;
  uint32_t nseg;
};

// Queue items: (graph << 44) | (iteration << 32) | segment.
constexpr unsigned long long kQueueEmpty = ~0ull;

struct BatchArgs {
  const BatchGraph *graphs;
  uint32_t ngraphs;
  unsigned long long *queue;      // ring of items
  uint32_t cap;                   // ring capacity (> items of one iteration of every graph)
  unsigned long long *head, *tail;
  uint32_t *active;               // graphs still running
  uint32_t *done_items;           // per graph: items finished in its current iteration
  unsigned long long *changed;    // per graph: changed count of its current iteration
  uint32_t *iters;                // per graph: iterations finished
  uint32_t *err;
  uint32_t max_iter;
  int early_exit;
  uint32_t cms_thr;
  uint32_t seeds[kCmsDepth];
  uint32_t *gtab;
  uint32_t gtab_slots;
  unsigned long long spin_limit;  // bound on the wait for an empty queue
};

__global__ void k_batch(BatchArgs b);
__global__ void k_batch_init(const BatchGraph *graphs, uint32_t ngraphs);

__global__ void k_iterate(IterArgs a);
// kGather: the cache path of the residual label reads (lpa_tune.gather_cache);
// kStage: the stream staging (lpa_tune.stage_stream); kPack: staged ids carry
// their lane (n <= 2^27, unstaged forms)
template <int kGather, int kStage, bool kPack>
__global__ void k_decode_two_pass(IterArgs a);
// V2 for tiny vertices: a lane per vertex.
__global__ void k_packed(IterArgs a);
// Two-pass variant, pass 2: counts the labels the pre-pass wrote.
// kBulk: group items staged by bulk copies (lpa_tune.bulk_stage)
template <bool kBulk>
__global__ void k_count_two_pass(IterArgs a);

// The template forms of the two-pass kernels are launched and sized only in
// the file that defines them (lp_kernels.cu):
// k_decode_two_pass<gather_cache, stage_stream, pack> on `grid` blocks of kThreads;
void launch_decode_two_pass(uint32_t gather_cache, uint32_t stage, int grid, cudaStream_t s, const IterArgs &a);
// k_count_two_pass<bulk> on `grid` blocks of kThreads with kCountSmemBytes;
void launch_count_two_pass(bool bulk, int grid, cudaStream_t s, const IterArgs &a);
// allows the stage_stream 2 forms their dynamic shared memory (once per device)
cudaError_t prepare_decode_two_pass();
// the fewest resident blocks per SM over each kernel's forms.
cudaError_t occupancy_decode_two_pass(int *blocks);
cudaError_t occupancy_count_two_pass(int *blocks);

struct DecodeArgs {
  DevGraph g;
  const uint32_t *pos_list;  // positions to decode (nullptr: [pos_begin, pos_begin + n_pos))
  uint64_t n_pos;
  uint64_t pos_begin;
  const uint64_t *arc_off;   // output offsets by position
  uint32_t *out;             // ids
  uint32_t *err;
};
__global__ void k_decode_positions(DecodeArgs a);

// Per compressed position: where its interval and residual sections'
// segments start (relative to its bit offset) and how many each has.
// Positions [p_lo, p_hi) (compressed ones only).
__global__ void k_pos_index(DevGraph g, uint4 *pidx, uint32_t *err, uint64_t p_lo, uint64_t p_hi);

// Degrees (and interval items) of positions [p_lo, p_hi).
__global__ void k_degree_count(DevGraph g, uint32_t *deg_out, uint32_t *itv_out, uint32_t *err, uint64_t p_lo,
                               uint64_t p_hi);
__global__ void k_init_labels(uint32_t *a, uint32_t *b, uint64_t n);

}  // namespace lpa_dev
