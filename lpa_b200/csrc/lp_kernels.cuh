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
  kVarBlock = 2,    // V3: block-per-vertex, segment-parallel decode, block table / sketch
  kVarTwoPass = 3,  // V4: decode to a CSR scratch, then count from it
  kNumVariants = 4
};

constexpr int kLaneWarps = 8;        // warps per block in the lane-batch kernel
constexpr uint32_t kStage = 1024;    // staged neighbour ids per warp
constexpr uint32_t kV1Slots = 512;   // exact-count table slots per warp (V1)
constexpr uint32_t kV1MaxDeg = kV1Slots / 2;
constexpr uint32_t kV2MaxDeg = 32;
constexpr int kBlockThreads = 256;   // V3 block size
constexpr uint32_t kBlockSlots = 8192;  // V3 shared exact-count table slots
constexpr uint32_t kBlockMaxSmemDeg = kBlockSlots / 2;

struct Seg {
  uint32_t begin, end;  // positions [begin, end)
};

struct IterArgs {
  DevGraph g;
  uint32_t *labs0, *labs1;      // the two label buffers
  uint32_t parity0;             // iteration 0 of this launch reads labs0 when 0, labs1 when 1
  const uint32_t *it_dev;       // device iteration counter (CUDA-graph loop), nullptr: 0
  unsigned long long *changed;  // changed counters, indexed by the iteration counter
  uint32_t *err;
  const Seg *segs;              // all segments
  const uint32_t *seg_list;     // segments handled by this launch
  uint32_t n_list;
  long long *seg_cycles;        // per-segment device cycles (nullptr: off)
  uint32_t cms_thr;             // 0: no sketch
  uint32_t seeds[kCmsDepth];
  // two-pass scratch: ids of compressed position p at scratch[arc_off[p]..)
  const uint32_t *scratch;
  const uint64_t *arc_off;
  int from_scratch;             // count from the scratch instead of decoding
  // global exact-count tables for V3 vertices above kBlockMaxSmemDeg
  uint32_t *gtab;
  uint32_t gtab_slots;          // slots per block (power of two), 0: none
};

// Resolves this launch's input/output buffers and changed counter.
__device__ __forceinline__ void resolve_iter(const IterArgs &a, const uint32_t *&lab_in, uint32_t *&lab_out,
                                             unsigned long long *&changed) {
  const uint32_t it = a.it_dev ? *a.it_dev : 0u;
  const uint32_t par = (a.parity0 + it) & 1u;
  lab_in = par ? a.labs1 : a.labs0;
  lab_out = par ? a.labs0 : a.labs1;
  changed = a.changed + (a.it_dev ? it : 0u);
}

__global__ void k_lane_batch_packed(IterArgs a);
__global__ void k_lane_batch_warp(IterArgs a);
__global__ void k_block(IterArgs a);

struct DecodeArgs {
  DevGraph g;
  const uint32_t *pos_list;  // positions to decode (nullptr: all of [0, n_pos))
  uint64_t n_pos;
  const uint64_t *arc_off;   // output offsets by position
  uint32_t *out;             // ids
  uint32_t *err;
};
__global__ void k_decode_positions(DecodeArgs a);
__global__ void k_decode_segments(IterArgs a);

__global__ void k_degree_count(DevGraph g, uint32_t *deg_out, uint32_t *err);
__global__ void k_init_labels(uint32_t *a, uint32_t *b, uint64_t n);

}  // namespace lpa_dev
