// Work lists of a plan, built on the device.
//
// A plan (one kernel variant per segment) becomes the kernels' work lists:
// k_iterate's heavy and light items, k_packed's chunks, the two-pass
// pre-pass's decode groups and the count pass's block, warp and group items
// (lp_kernels.cuh).  Building them is a walk over every segment's positions.
// Here one thread walks one segment (at most 256 positions, or one hub), twice:
// once to count its items, and after an exclusive scan of the counts once more
// to write them at their offsets.  The count pass's group items (up to
// group_positions consecutive positions of degree <= 32) run across segments
// and across isolated vertices, so they are formed per aligned window of
// group_positions positions instead: a window's item is a run of such
// positions (isolated ones between them included), trimmed to its first and
// last counted position.  Heavy items and the count pass's block items are
// then sorted largest first by a stable radix sort (CUB, from the CUDA
// toolkit), so the largest work starts first.  A plan change -- a learner
// trial, an autotuner candidate, lpa_set_plan -- thus costs a few launches
// and one small copy of the list sizes back to the host, not a host loop over
// every position (baselines/novaplus/novaplus_propogator.cuh:208-304 builds
// its tiny-vertex assignment on the host).
#include <cuda_runtime.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <string>
#include <vector>

#include "plan.cuh"

namespace lpa_dev {

namespace {

enum List : int { kLHeavy = 0, kLLight, kLPacked, kLGroups, kLBlock, kLWarp, kLists };

struct PlanArgs {
  const SegDev *segs;
  uint32_t seg_begin, nseg;
  const uint8_t *var;
  const uint32_t *deg;       // by position
  const uint32_t *vertices;  // by position
  const uint4 *pidx;         // per compressed position (two-pass plans only)
  const uint64_t *arc_off;   // n + 1 (two-pass plans only)
  const uint64_t *offsets;   // n_c + 1
  const uint32_t *small_off; // n - n_c + 1
  const uint32_t *words, *small_nbr, *scratch;
  uint64_t n, n_c;
  uint32_t cms, wmax, warp_positions, group_positions;
  uint64_t c_begin, c_end, s_begin, s_end;  // positions of the group items (compressed, small CSR)
  uint64_t win0;             // windows of the compressed positions; the rest cover the small CSR
  const uint32_t *off;       // kLists x (nseg + 1) exclusive offsets, by segment - seg_begin
  uint32_t *cnt;             // kLists x (nseg + 1) counts
  uint32_t *gmark;           // n: 1 + segment of a position counted by a group item, else 0
  uint32_t *win_cnt;         // per window: group items
  const uint32_t *win_off;
  // outputs
  WorkItem *heavy;           // unsorted, with keys
  uint32_t *heavy_key;
  WorkItem *light;
  PackedChunk *packed;
  DecodeGroup *groups;
  BlockItem *cblock;         // unsorted, with keys
  uint32_t *cblock_key;
  CountItem *cwarp;          // warp items, then group items from n_warp on
  uint32_t n_warp;
};

__device__ __forceinline__ bool warp_capable(const SegDev &si, uint32_t cms) {
  return !(cms != 0 && si.max_deg >= cms) && si.max_deg <= kV1MaxDeg;
}

// The device range a work item over positions [p0, p1) will read (for its
// L2 prefetch): the bitstream words, the scratch labels or the small-CSR ids.
__device__ WorkItem make_item(const PlanArgs &a, uint32_t tag, uint32_t p0, uint32_t p1, bool two_pass) {
  uint64_t addr = 0, bytes = 0;
  if (p0 < a.n_c) {
    if (two_pass) {
      addr = reinterpret_cast<uint64_t>(a.scratch + a.arc_off[p0]);
      bytes = (a.arc_off[p1] - a.arc_off[p0]) * 4;
    } else {
      const uint64_t b = a.offsets[p0] >> 5, e = a.offsets[p1] >> 5;
      addr = reinterpret_cast<uint64_t>(a.words + b);
      bytes = (e - b + 3) * 4;
    }
  } else {
    const uint64_t b = a.small_off[p0 - a.n_c], e = a.small_off[p1 - a.n_c];
    addr = reinterpret_cast<uint64_t>(a.small_nbr + b);
    bytes = (e - b) * 4;
  }
  return WorkItem{tag, uint32_t(bytes < 0x7FFFFFFFull ? bytes : 0x7FFFFFFFull), addr};
}

// One segment's items.  kEmit false: counts them (and marks the positions
// its group items will take); true: writes them at the scanned offsets.
template <bool kEmit>
__device__ void plan_segment(const PlanArgs &a, uint32_t i) {
  const uint32_t s = a.seg_begin + i;
  const SegDev si = a.segs[s];
  const int v = a.var[s];
  const uint32_t cms = a.cms;
  const bool tp = v == kVarTwoPass;
  // a block-variant segment whose vertices one warp holds runs as warp
  // chunks (one vertex per warp at a time, k_iterate's light loop) instead of
  // one vertex per block: its vertices have at most 64 segments of 256 bits,
  // too few to keep a block busy, and block items wait at barriers
  const bool block = (v == kVarBlock || tp) && !warp_capable(si, cms);
  bool counted = tp;  // the two-pass count pass takes the segment's positions
  if (tp) {
    // exact above the count pass's block table (a hub is alone in its segment)
    if (si.max_deg > kCountBlockMax && (cms == 0 || si.max_deg < cms)) counted = false;
    // the small CSR is counted by warp and group items only
    if (si.region == 1 && ((cms != 0 && si.max_deg >= cms) || si.max_deg > a.wmax)) counted = false;
  }
  const uint32_t stride = a.nseg + 1;
  uint32_t c[kLists] = {0, 0, 0, 0, 0, 0};
  uint32_t o[kLists] = {0, 0, 0, 0, 0, 0};
  if (kEmit)
    for (int l = 0; l < kLists; l++) o[l] = a.off[l * stride + i];
  if (counted) {
    uint32_t p = si.begin;
    while (p < si.end) {
      const uint32_t d = a.deg[p];
      const bool sk = cms != 0 && d >= cms;
      if (sk || d > a.wmax) {
        if (kEmit) {
          const uint32_t at = o[kLBlock] + c[kLBlock];
          a.cblock[at] = BlockItem{a.arc_off[p], p, d, a.vertices[p], s,
                                   sk ? uint32_t(kCountSketch) : uint32_t(kCountBlock), 0u};
          a.cblock_key[at] = d;
        }
        c[kLBlock]++;
        p++;
      } else if (d <= 32) {
        if (!kEmit) a.gmark[p] = s + 1;
        p++;
      } else {
        uint32_t q = p + 1;
        while (q < si.end && q - p < a.warp_positions) {
          const uint32_t dq = a.deg[q];
          if ((cms != 0 && dq >= cms) || dq > a.wmax || dq <= 32) break;
          q++;
        }
        if (kEmit) a.cwarp[o[kLWarp] + c[kLWarp]] = CountItem{p, q - p, s, uint32_t(kCountWarp)};
        c[kLWarp]++;
        p = q;
      }
    }
  } else if (block) {
    if (kEmit) {
      a.heavy[o[kLHeavy]] = make_item(a, s, si.begin, si.end, tp);
      a.heavy_key[o[kLHeavy]] = uint32_t(si.arcs < 0xFFFFFFFFull ? si.arcs : 0xFFFFFFFFull);
    }
    c[kLHeavy] = 1;
  } else if (v == kVarPacked && si.max_deg <= kPackedMaxDeg) {
    for (uint32_t p0 = si.begin; p0 < si.end; p0 += 32) {
      if (kEmit) a.packed[o[kLPacked] + c[kLPacked]] = PackedChunk{p0, min(si.end - p0, 32u), s, 0u};
      c[kLPacked]++;
    }
  } else {
    const uint32_t chunks = (si.end - si.begin + 31) / 32;
    for (uint32_t k = 0; k < chunks; k++) {
      const uint32_t p0 = si.begin + 32 * k, p1 = min(si.end, p0 + 32);
      if (kEmit) a.light[o[kLLight] + k] = make_item(a, (s << 3) | k, p0, p1, tp);
    }
    c[kLLight] = chunks;
  }
  if (tp && si.region == 0) {
    // decode groups: 32 consecutive 256-bit segments of the positions,
    // spanning at most 32 positions
    // first bit of segment j of position q (interval segments first)
    const auto seg_bit = [&](uint32_t q, uint32_t jq, const uint4 &ix) {
      return a.offsets[q] + (jq < ix.z ? uint64_t(ix.x) + uint64_t(kSegBits) * jq
                                       : uint64_t(ix.y) + uint64_t(kSegBits) * (jq - ix.z));
    };
    uint32_t p = si.begin, j = 0;
    while (p < si.end) {
      DecodeGroup gd{p, j, 0u, s, 0ull, 0u, 0u};
      const uint64_t first = seg_bit(p, j, a.pidx[p]);
      uint32_t positions = 0, lp = p, lj = j;
      while (p < si.end && gd.nlanes < 32 && positions < 32) {
        const uint4 ix = a.pidx[p];
        const uint32_t ns = ix.z + ix.w;
        const uint32_t take = min(ns - j, 32u - gd.nlanes);
        gd.nlanes += take;
        positions++;
        if (take) {
          lp = p;
          lj = j + take - 1;
        }
        if (j + take == ns) {
          p++;
          j = 0;
        } else {
          j += take;
        }
      }
      // the span its lanes read: from the first segment to the end of the
      // last (a section's last segment is under 512 bits), plus the 2 words
      // a reader loads ahead
      const uint64_t last_end = min(a.offsets[lp + 1], seg_bit(lp, lj, a.pidx[lp]) + 2 * kSegBits);
      gd.w0 = first >> 5;
      const uint64_t wn = (last_end >> 5) + 3 - gd.w0;
      gd.wn = uint32_t(wn < 0xFFFFFFFFull ? wn : 0xFFFFFFFFull);
      if (gd.nlanes) {
        if (kEmit) a.groups[o[kLGroups] + c[kLGroups]] = gd;
        c[kLGroups]++;
      }
    }
  }
  if (!kEmit)
    for (int l = 0; l < kLists; l++) a.cnt[l * stride + i] = c[l];
}

__global__ void k_plan_count(PlanArgs a) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nseg; i += gridDim.x * blockDim.x)
    plan_segment<false>(a, i);
}

__global__ void k_plan_emit(PlanArgs a) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.nseg; i += gridDim.x * blockDim.x)
    plan_segment<true>(a, i);
}

// Group items of one window: runs of marked or isolated positions, trimmed
// to their marked ends.  Windows of the compressed region come first.
template <bool kEmit>
__device__ void plan_window(const PlanArgs &a, uint64_t w) {
  const uint64_t G = a.group_positions;
  uint64_t w0, w1;
  if (w < a.win0) {
    w0 = a.c_begin + w * G;
    w1 = min(w0 + G, a.c_end);
  } else {
    w0 = a.s_begin + (w - a.win0) * G;
    w1 = min(w0 + G, a.s_end);
  }
  uint32_t k = 0;
  const uint32_t at = kEmit ? a.n_warp + a.win_off[w] : 0u;
  uint64_t p = w0;
  while (p < w1) {
    const uint32_t m = a.gmark[p];
    if (!m) {
      p++;
      continue;
    }
    uint64_t q = p + 1, last = p;
    while (q < w1) {
      const uint32_t mq = a.gmark[q];
      if (mq) last = q;
      else if (a.deg[q] != 0) break;
      q++;
    }
    if (kEmit) a.cwarp[at + k] = CountItem{uint32_t(p), uint32_t(last + 1 - p), m - 1, uint32_t(kCountGroups)};
    k++;
    p = last + 1;
  }
  if (!kEmit) a.win_cnt[w] = k;
}

__global__ void k_window_count(PlanArgs a, uint64_t nwin) {
  for (uint64_t w = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; w < nwin; w += uint64_t(gridDim.x) * blockDim.x)
    plan_window<false>(a, w);
}

__global__ void k_window_emit(PlanArgs a, uint64_t nwin) {
  for (uint64_t w = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; w < nwin; w += uint64_t(gridDim.x) * blockDim.x)
    plan_window<true>(a, w);
}

// The list sizes: offset[nseg] of every list, then the group items.
__global__ void k_plan_totals(const uint32_t *off, uint32_t stride, const uint32_t *win_off, uint64_t nwin,
                              uint32_t *tot) {
  if (threadIdx.x < kLists) tot[threadIdx.x] = off[threadIdx.x * stride + stride - 1];
  if (threadIdx.x == kLists) tot[kLists] = win_off[nwin];
}

template <class T>
__global__ void k_gather(const T *src, const uint32_t *idx, T *dst, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

__global__ void k_iota(uint32_t *x, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] = i;
}

int grid_for(uint64_t work, int num_sms) {
  return int(std::max<uint64_t>(1, std::min<uint64_t>((work + 255) / 256, uint64_t(num_sms) * 16)));
}

}  // namespace

void PlanBuilder::release() {
  for (void *p : bufs)
    if (p) cudaFree(p);
  bufs.clear();
  *this = PlanBuilder{};
}

cudaError_t PlanBuilder::reserve(void **ptr, size_t &cap, size_t bytes) {
  if (*ptr && cap >= bytes) return cudaSuccess;
  if (*ptr) {
    bufs.erase(std::find(bufs.begin(), bufs.end(), *ptr));
    cudaFree(*ptr);
    *ptr = nullptr;
  }
  const size_t want = std::max<size_t>(256, bytes + bytes / 4);
  cudaError_t e = cudaMalloc(ptr, want);
  if (e != cudaSuccess) {
    *ptr = nullptr;
    cap = 0;
    return e;
  }
  bufs.push_back(*ptr);
  cap = want;
  return cudaSuccess;
}

cudaError_t PlanBuilder::build(const PlanInputs &in, PlanOutputs &out, cudaStream_t st, std::string &where) {
#define PB_TRY(call, what)            \
  do {                                \
    const cudaError_t e_ = (call);    \
    if (e_ != cudaSuccess) {          \
      where = what;                   \
      return e_;                      \
    }                                 \
  } while (0)
  const uint32_t S = in.nseg;
  const uint32_t stride = S + 1;
  const uint64_t G = std::max<uint32_t>(1, in.group_positions);
  const uint64_t win0 = (in.c_end - in.c_begin + G - 1) / G, win1 = (in.s_end - in.s_begin + G - 1) / G;
  const uint64_t nwin = win0 + win1;
  PB_TRY(reserve(reinterpret_cast<void **>(&cnt), cnt_cap, size_t(kLists) * stride * 4), "plan counts");
  PB_TRY(reserve(reinterpret_cast<void **>(&off), off_cap, size_t(kLists) * stride * 4), "plan offsets");
  PB_TRY(reserve(reinterpret_cast<void **>(&gmark), gmark_cap, std::max<uint64_t>(1, in.n) * 4), "group marks");
  PB_TRY(reserve(reinterpret_cast<void **>(&win), win_cap, (nwin + 1) * 4), "window counts");
  PB_TRY(reserve(reinterpret_cast<void **>(&win_off), win_off_cap, (nwin + 1) * 4), "window offsets");
  PB_TRY(reserve(reinterpret_cast<void **>(&tot), tot_cap, 8 * 4), "plan totals");
  PB_TRY(cudaMemsetAsync(cnt, 0, size_t(kLists) * stride * 4, st), "clear counts");
  PB_TRY(cudaMemsetAsync(win, 0, (nwin + 1) * 4, st), "clear windows");
  PB_TRY(cudaMemsetAsync(gmark, 0, std::max<uint64_t>(1, in.n) * 4, st), "clear marks");

  PlanArgs a{};
  a.segs = in.segs;
  a.seg_begin = in.seg_begin;
  a.nseg = S;
  a.c_begin = in.c_begin;
  a.c_end = in.c_end;
  a.s_begin = in.s_begin;
  a.s_end = in.s_end;
  a.var = in.var;
  a.deg = in.deg;
  a.vertices = in.vertices;
  a.pidx = in.pidx;
  a.arc_off = in.arc_off;
  a.offsets = in.offsets;
  a.small_off = in.small_off;
  a.words = in.words;
  a.small_nbr = in.small_nbr;
  a.scratch = in.scratch;
  a.n = in.n;
  a.n_c = in.n_c;
  a.cms = in.cms;
  a.wmax = in.wmax;
  a.warp_positions = in.warp_positions;
  a.group_positions = uint32_t(G);
  a.win0 = win0;
  a.off = off;
  a.cnt = cnt;
  a.gmark = gmark;
  a.win_cnt = win;
  a.win_off = win_off;
  if (S) k_plan_count<<<grid_for(S, in.num_sms), 256, 0, st>>>(a);
  PB_TRY(cudaGetLastError(), "plan count launch");
  if (nwin) k_window_count<<<grid_for(nwin, in.num_sms), 256, 0, st>>>(a, nwin);
  PB_TRY(cudaGetLastError(), "window count launch");
  // exclusive scans (one extra element each: its offset is the total)
  size_t need = 0, t = 0;
  PB_TRY(cub::DeviceScan::ExclusiveSum(nullptr, t, cnt, off, stride, st), "scan size");
  need = std::max(need, t);
  PB_TRY(cub::DeviceScan::ExclusiveSum(nullptr, t, win, win_off, nwin + 1, st), "scan size");
  need = std::max(need, t);
  PB_TRY(reserve(&temp, temp_cap, need), "scan temp");
  for (int l = 0; l < kLists; l++) {
    t = temp_cap;
    PB_TRY(cub::DeviceScan::ExclusiveSum(temp, t, cnt + size_t(l) * stride, off + size_t(l) * stride, stride, st),
           "scan");
  }
  t = temp_cap;
  PB_TRY(cub::DeviceScan::ExclusiveSum(temp, t, win, win_off, nwin + 1, st), "window scan");
  k_plan_totals<<<1, 32, 0, st>>>(off, stride, win_off, nwin, tot);
  PB_TRY(cudaGetLastError(), "totals launch");
  uint32_t h_tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  PB_TRY(cudaMemcpyAsync(h_tot, tot, 8 * 4, cudaMemcpyDeviceToHost, st), "read totals");
  PB_TRY(cudaStreamSynchronize(st), "plan totals");
  out.n_heavy = h_tot[kLHeavy];
  out.n_light = h_tot[kLLight];
  out.n_packed = h_tot[kLPacked];
  out.n_groups = h_tot[kLGroups];
  out.n_cblock = h_tot[kLBlock];
  out.n_cwarp = h_tot[kLWarp] + h_tot[kLists];

  // outputs (the caller's buffers grow to fit) and sort staging
  PB_TRY(out.grow(out), "work lists");
  const uint32_t nsort = std::max(out.n_heavy, out.n_cblock);
  PB_TRY(reserve(reinterpret_cast<void **>(&heavy_tmp), heavy_tmp_cap, size_t(out.n_heavy + 1) * sizeof(WorkItem)),
         "heavy staging");
  PB_TRY(reserve(reinterpret_cast<void **>(&cblock_tmp), cblock_tmp_cap,
                 size_t(out.n_cblock + 1) * sizeof(BlockItem)), "block staging");
  PB_TRY(reserve(reinterpret_cast<void **>(&keys), keys_cap, size_t(nsort + 1) * 4 * 4), "sort keys");
  a.heavy = heavy_tmp;
  a.heavy_key = keys;
  a.cblock = cblock_tmp;
  a.cblock_key = keys + (nsort + 1);
  a.light = out.items + out.n_heavy;
  a.packed = out.packed;
  a.groups = out.groups;
  a.cwarp = out.cwarp;
  a.n_warp = h_tot[kLWarp];
  if (S) k_plan_emit<<<grid_for(S, in.num_sms), 256, 0, st>>>(a);
  PB_TRY(cudaGetLastError(), "plan emit launch");
  if (nwin) k_window_emit<<<grid_for(nwin, in.num_sms), 256, 0, st>>>(a, nwin);
  PB_TRY(cudaGetLastError(), "window emit launch");

  // largest first, ties in segment order (a stable radix sort of the keys
  // with the item indices)
  uint32_t *kout = keys + 2 * (nsort + 1);
  uint32_t *idx_in = nullptr, *idx_out = nullptr;
  PB_TRY(reserve(reinterpret_cast<void **>(&idx), idx_cap, size_t(nsort + 1) * 2 * 4), "sort indices");
  idx_in = idx;
  idx_out = idx + (nsort + 1);
  auto sort_gather = [&](const uint32_t *k_in, uint32_t count, auto *src, auto *dst) -> cudaError_t {
    if (count == 0) return cudaSuccess;
    k_iota<<<grid_for(count, in.num_sms), 256, 0, st>>>(idx_in, count);
    size_t sb = 0;
    cudaError_t e = cub::DeviceRadixSort::SortPairsDescending(nullptr, sb, k_in, kout, idx_in, idx_out, count, 0, 32, st);
    if (e != cudaSuccess) return e;
    e = reserve(&temp, temp_cap, sb);
    if (e != cudaSuccess) return e;
    sb = temp_cap;
    e = cub::DeviceRadixSort::SortPairsDescending(temp, sb, k_in, kout, idx_in, idx_out, count, 0, 32, st);
    if (e != cudaSuccess) return e;
    k_gather<<<grid_for(count, in.num_sms), 256, 0, st>>>(src, idx_out, dst, count);
    return cudaGetLastError();
  };
  PB_TRY(sort_gather(keys, out.n_heavy, heavy_tmp, out.items), "sort heavy items");
  PB_TRY(sort_gather(keys + (nsort + 1), out.n_cblock, cblock_tmp, out.cblock), "sort block items");
  return cudaSuccess;
#undef PB_TRY
}

}  // namespace lpa_dev
