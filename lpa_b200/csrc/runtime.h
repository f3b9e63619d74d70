// Internal runtime structures behind the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "lp_kernels.cuh"
#include "lpa_capi.h"
#include "plan.cuh"

namespace lpa_rt {

// Degree buckets used to cut segments (the reference's buckets,
// baselines/novaplus/novaplus_propogator.cuh:219-220, plus a "heavy" bucket
// for vertices only the block and two-pass variants can take).
enum Bucket : uint8_t { kTiny = 0, kMid = 1, kLarge = 2, kHeavy = 3, kNumBuckets = 4 };


struct SegInfo {
  uint32_t begin, end;
  uint8_t bucket;
  uint8_t region;  // 0: compressed, 1: small CSR
  uint32_t max_deg;
  uint64_t arcs;
  uint64_t bits;
  uint32_t intervals;  // interval count (features)
};

struct CudaError {
  cudaError_t e;
  const char *where;
};

inline uint32_t next_pow2_host(uint64_t x) {
  uint32_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

bool variant_capable(int variant, const SegInfo &s, uint32_t cms_thr);
int fixed_variant(const SegInfo &s);
// Segments of a graph from its degrees by position (runs of one bucket).
std::vector<SegInfo> make_segments(const uint32_t *deg, uint64_t n, uint64_t n_c, uint32_t cms_thr);

}  // namespace lpa_rt

// One range of an out-of-core (streamed) handle: compressed positions
// [p0, p1) and the plan segments [s0, s1) inside them (the last range also
// takes the small CSR's segments), the stream words [w0, w1) they read and
// their two-pass scratch indices [a0, a1), with the range's own work lists.
struct StreamRange {
  uint64_t p0 = 0, p1 = 0;
  uint32_t s0 = 0, s1 = 0;
  uint64_t w0 = 0, w1 = 0;
  uint64_t a0 = 0, a1 = 0;
  bool last = false;
  lpa_dev::WorkItem *items = nullptr;
  lpa_dev::PackedChunk *packed = nullptr;
  lpa_dev::DecodeGroup *groups = nullptr;
  lpa_dev::BlockItem *cblock = nullptr;
  lpa_dev::CountItem *cwarp = nullptr;
  size_t items_cap = 0, packed_cap = 0, groups_cap = 0, cblock_cap = 0, cwarp_cap = 0;
  uint32_t n_heavy = 0, n_light = 0, n_packed = 0, n_groups = 0, n_cblock = 0, n_cwarp = 0;
  int grid_decode = 1;
};

struct lpa_handle {
  lpa_opts opts{};
  lpa_tune tune{32, 4, lpa_dev::kCountWarpMax, 2, 0, 0, 0};  // count-pass work shapes (lpa_set_tune / lpa_autotune)
  bool measure_busy = false;                        // record kernel busy spans (IterArgs::ktime)
  bool learner_spans = false;                       // the same, for the learned dispatch's iteration clock
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  std::string last_error;
  int num_sms = 148;

  uint64_t n = 0, n_c = 0, nwords = 0, m_small = 0, m = 0, total_bits = 0, max_deg = 0;
  uint32_t seeds[lpa_dev::kCmsDepth] = {0, 0, 0, 0};

  // device graph
  uint32_t *d_words = nullptr, *d_vertices = nullptr, *d_deg = nullptr;
  uint32_t *d_small_off = nullptr, *d_small_nbr = nullptr;
  uint64_t *d_offsets = nullptr;
  uint32_t *d_lab[2] = {nullptr, nullptr};
  int cur = 0;
  unsigned long long *d_changed = nullptr;  // one slot per iteration of a run
  int changed_slots = 0;
  uint32_t *d_err = nullptr;
  unsigned long long *h_pinned = nullptr;  // pinned readback

  // plan
  std::vector<uint32_t> h_deg;
  std::vector<lpa_rt::SegInfo> segs;
  std::vector<uint8_t> variant;  // per segment
  std::vector<uint8_t> fixed;    // per segment, the heuristic's choice
  lpa_dev::Seg *d_segs = nullptr;
  lpa_dev::SegDev *d_segdev = nullptr;       // the segments as the device list builder reads them
  lpa_dev::PlanBuilder plan_builder;         // its working memory
  uint8_t *d_seg_var = nullptr;
  lpa_dev::WorkItem *d_items = nullptr;  // heavy items | light chunk items
  lpa_dev::DecodeGroup *d_groups = nullptr;  // two-pass pre-pass work (32 segments each)
  uint32_t n_heavy = 0, n_light = 0, n_groups = 0;
  size_t items_cap = 0, groups_cap = 0;
  uint4 *d_pidx = nullptr;                   // per compressed position: section starts and segment counts
  uint32_t *d_cursor = nullptr;              // per compressed position: pre-pass output cursor
  lpa_dev::CountItem *d_citems = nullptr;    // count-pass warp items
  lpa_dev::BlockItem *d_cblock = nullptr;    // count-pass block items
  lpa_dev::PackedChunk *d_packed = nullptr;  // k_packed work
  uint32_t n_packed = 0;
  size_t packed_cap = 0;
  int grid_packed = 0;
  uint32_t cw_packed = 1;
  size_t cblock_cap = 0;
  uint32_t n_cblock = 0, n_cwarp = 0;
  size_t citems_cap = 0;
  int grid_count = 0;                        // count-pass kernel
  uint32_t cw_iterate = 1, cw_decode = 1, cw_count = 1;  // seg_cycles weights (64 / resident warps per SM)
  std::vector<uint64_t> h_arc_off;
  int grid = 0;          // persistent iteration kernel
  int grid_decode = 0;   // two-pass decode kernel
  int occ = 1;
  int occ_decode = 1;    // resident blocks per SM of the two-pass decode kernel
  uint32_t *d_work = nullptr;        // kWorkCounters queue counters per iteration slot
  uint32_t *d_seg_changed = nullptr; // per-segment changed counts (cost-model feature)
  uint32_t *d_seg_changed_prev = nullptr;  // the previous iteration's

  // scratch
  uint64_t *d_arc_off = nullptr;
  uint32_t *d_scratch = nullptr;
  uint32_t *d_gtab = nullptr;
  uint32_t *d_hub_spill = nullptr;  // per block of k_iterate: a sketch hub's labels (second pass)
  uint32_t hub_spill_words = 0;
  uint32_t max_sketch_deg = 0;      // largest degree at or above the sketch threshold
  uint32_t gtab_slots = 0;
  int gtab_blocks = 0;
  long long *d_seg_cycles = nullptr;
  unsigned long long *d_ktime = nullptr;  // busy span of each kernel of a learning iteration (IterArgs::ktime)

  // stats
  uint64_t iterations = 0;
  uint64_t launches = 0;
  uint64_t last_changed = 0;
  std::vector<uint64_t> history;
  double last_iter_ms = 0;
  double variant_ms[4] = {0, 0, 0, 0};
  double decode_ms = 0, iterate_ms = 0, count_ms = 0, packed_ms = 0;
  bool collect_cycles = false;  // per-segment cycles for the cost model
  cudaEvent_t ev[5] = {};  // iteration start, then one after each kernel that ran
  int ev_kernel[5] = {};   // which kernel each event follows (0 pre-pass, 1 count, 2 k_packed, 3 k_iterate)
  int ev_used = 0;
  bool events_ready = false;
  uint64_t device_bytes = 0;
  std::vector<void *> allocations;

  // out-of-core streaming (opts.stream_budget): the stream in pinned host
  // memory, two device buffers filled on copy_stream, the ranges
  bool streamed = false;
  uint32_t *h_wpinned = nullptr;
  uint32_t *d_wbuf[2] = {nullptr, nullptr};
  uint64_t wbuf_words = 0;     // capacity of each buffer (words)
  uint64_t scratch_words = 0;  // capacity of the streamed scratch (words)
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_ready[2] = {}, ev_free[2] = {};
  std::vector<StreamRange> ranges;
  uint64_t streamed_bytes = 0;  // stream bytes copied host -> device so far
  int wbuf_range[2] = {-1, -1};  // the range whose words each buffer holds (-1: none)
  const uint64_t *create_offsets = nullptr;  // the caller's bit offsets, during lpa_create only

  // CUDA-graph loop: while set, kernels take their parity and counter slot from it
  const uint32_t *loop_it = nullptr;
  uint32_t *d_loop_it = nullptr;
  void *graph_exec = nullptr;  // cudaGraphExec_t of the early-exit loop
  void *graph = nullptr;       // cudaGraph_t
  uint64_t launches_per_graph_iteration = 0;
  uint64_t plan_version = 0, graph_plan_version = ~0ull;

  // learned dispatch (cost model), see dispatch.cu
  struct Learner *learner = nullptr;

  // graphs concatenated into this one (a lockstep batch, batch.cu): graph k
  // owns vertex ids [d_gbase[k], d_gbase[k + 1]).  d_gtrack: [0] iterations
  // done, [1] max_iter, [2] early exit, [3] unused, then n_graphs changed
  // flags, then n_graphs iteration counts (0: still running)
  uint32_t *d_gbase = nullptr;
  uint32_t n_graphs = 0;
  uint32_t *d_gtrack = nullptr;
};

// Hooks between the runtime modules (C++ linkage).
void lpa_rt_destroy_graph(lpa_handle *h);
lpa_status lpa_run_graph(lpa_handle *h, int max_iter, bool early_exit, int *iters_done);
void lpa_learner_free(lpa_handle *h);
void lpa_learner_reset(lpa_handle *h);
void lpa_learner_before_iteration(lpa_handle *h);
void lpa_learner_after_iteration(lpa_handle *h);
void lpa_learner_stats(lpa_handle *h, lpa_stats *st);
bool lpa_learner_settled(lpa_handle *h);
void lpa_rt_enqueue_iteration(lpa_handle *h, unsigned long long *changed, uint32_t *work);
// Per-graph convergence of a lockstep batch, enqueued after every iteration
// (2 launches).
void lpa_rt_enqueue_track(lpa_handle *h);
void lpa_rt_apply_variants(lpa_handle *h);
lpa_status lpa_rt_take_error(lpa_handle *h);
