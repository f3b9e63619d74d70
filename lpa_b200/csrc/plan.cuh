// Device-built work lists of a plan (plan.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <string>
#include <vector>

#include "lp_kernels.cuh"

namespace lpa_dev {

// A segment as the list builder reads it.
struct SegDev {
  uint32_t begin, end;  // positions [begin, end)
  uint32_t max_deg;
  uint8_t bucket, region, pad0, pad1;
  uint64_t arcs;
};

struct PlanInputs {
  const SegDev *segs;        // every segment of the graph
  uint32_t seg_begin;        // the lists cover segments [seg_begin, seg_begin + nseg)
  uint32_t nseg;
  // and the count pass's group items positions [c_begin, c_end) of the
  // compressed region and [s_begin, s_end) of the small CSR
  uint64_t c_begin, c_end, s_begin, s_end;
  const uint8_t *var;        // variant per segment
  const uint32_t *deg;       // degree by position
  const uint32_t *vertices;  // vertex id by position
  const uint4 *pidx;         // position index (two-pass plans), else nullptr
  const uint64_t *arc_off;   // scratch offsets (two-pass plans), else nullptr
  const uint64_t *offsets;   // bit offsets, n_c + 1
  const uint32_t *small_off; // small CSR offsets, n - n_c + 1
  const uint32_t *words, *small_nbr, *scratch;
  uint64_t n, n_c;
  uint32_t cms;              // sketch threshold (0: none)
  uint32_t wmax;             // lpa_tune.warp_max_degree
  uint32_t warp_positions;   // lpa_tune.warp_positions
  uint32_t group_positions;  // lpa_tune.group_positions
  int num_sms;
};

// The lists, in the caller's device buffers.  build() sets the counts, then
// calls grow(), which must make the buffers hold them (it may reallocate),
// then writes the lists: items = heavy items (largest first) followed by
// light items; cwarp = warp items followed by group items; cblock largest
// first.
struct PlanOutputs {
  uint32_t n_heavy = 0, n_light = 0, n_packed = 0, n_groups = 0, n_cblock = 0, n_cwarp = 0;
  WorkItem *items = nullptr;
  PackedChunk *packed = nullptr;
  DecodeGroup *groups = nullptr;
  BlockItem *cblock = nullptr;
  CountItem *cwarp = nullptr;
  std::function<cudaError_t(PlanOutputs &)> grow;
};

// Working memory of the builder, kept between plan changes of one handle.
class PlanBuilder {
 public:
  // Enqueues the build on st; waits once for the list sizes.  On failure
  // `where` names the step.
  cudaError_t build(const PlanInputs &in, PlanOutputs &out, cudaStream_t st, std::string &where);
  void release();

 private:
  cudaError_t reserve(void **ptr, size_t &cap, size_t bytes);
  std::vector<void *> bufs;
  uint32_t *cnt = nullptr, *off = nullptr, *gmark = nullptr, *win = nullptr, *win_off = nullptr, *tot = nullptr;
  uint32_t *keys = nullptr, *idx = nullptr;
  WorkItem *heavy_tmp = nullptr;
  BlockItem *cblock_tmp = nullptr;
  void *temp = nullptr;
  size_t cnt_cap = 0, off_cap = 0, gmark_cap = 0, win_cap = 0, win_off_cap = 0, tot_cap = 0, keys_cap = 0,
         idx_cap = 0, heavy_tmp_cap = 0, cblock_tmp_cap = 0, temp_cap = 0;
};

}  // namespace lpa_dev
