// Declarations shared by noalloc.cu and the kernels in noalloc_kernels.cuh.
#pragma once
#include "lp_kernels.cuh"

namespace lpa_dev {

// ---- one two-pass iteration over caller-owned device buffers ------------
// The decoded CSR, the per-position degrees and offsets and the counters live
// in the library's static device array (g_noalloc_scratch in noalloc.cu), not
// in caller memory.
struct NoAllocArgs {
  DevGraph g;                   // g.deg points into the scratch region
  uint32_t *deg;                // n degrees by position
  uint64_t *arc_off;            // n_c + 1 offsets into ids
  uint32_t *ids;                // decoded ids of the compressed positions
  unsigned long long *stats;    // [0] changed, [1] max degree, [2] arcs of compressed positions
  uint32_t *err;
  const uint32_t *lab_in;
  uint32_t *lab_out;
  uint32_t cms_thr;
  uint64_t total_bits;          // offsets[n_c]: every vertex's bits must lie below it
  uint64_t small_arcs;          // small-CSR ids available
};
__global__ void k_na_degrees(NoAllocArgs a);
__global__ void k_na_scan(NoAllocArgs a);
__global__ void k_na_decode(NoAllocArgs a);
__global__ void k_na_count(NoAllocArgs a);

}  // namespace lpa_dev
