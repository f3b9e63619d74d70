// C ABI implementation: device graph, dispatch plan and the iteration loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <cstring>
#include <new>
#include <string>
#include <type_traits>
#include <vector>

#include "lp_kernels.cuh"
#include "lpa_capi.h"
#include "plan.cuh"
#include "runtime.h"

using namespace lpa_dev;
using namespace lpa_rt;

namespace {

constexpr int kMaxRunSlots = 1 << 16;

// Segment cutting limits per bucket: positions (light segments hold at most
// 8 warp chunks of 32) and arcs.
constexpr uint32_t kSegPositions[kNumBuckets] = {256, 256, 64, 1};
constexpr uint64_t kSegArcs = 16384;

struct Fail {
  lpa_status st;
  std::string msg;
};

void check(lpa_handle *h, cudaError_t e, const char *where) {
  if (e != cudaSuccess) {
    lpa_status st = (e == cudaErrorMemoryAllocation) ? LPA_ERR_OOM : LPA_ERR_CUDA;
    throw Fail{st, std::string(where) + ": " + cudaGetErrorString(e)};
  }
  (void)h;
}

template <class T>
T *dalloc(lpa_handle *h, uint64_t count, const char *what) {
  void *p = nullptr;
  const uint64_t bytes = std::max<uint64_t>(count, 1) * sizeof(T);
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Fail{LPA_ERR_OOM, std::string("cudaMalloc ") + what + " (" + std::to_string(bytes) + " bytes)"};
  }
  h->allocations.push_back(p);
  h->device_bytes += bytes;
  return static_cast<T *>(p);
}

template <class T>
void h2d(lpa_handle *h, T *dst, const T *src, uint64_t count, const char *what) {
  if (count == 0) return;
  check(h, cudaMemcpyAsync(dst, src, count * sizeof(T), cudaMemcpyHostToDevice, h->stream), what);
}

lpa_status guard(lpa_handle *h, const Fail &f) {
  if (h) h->last_error = f.msg;
  return f.st;
}

DevGraph dev_graph(const lpa_handle *h) {
  DevGraph g;
  g.words = h->d_words;
  g.offsets = h->d_offsets;
  g.vertices = h->d_vertices;
  g.deg = h->d_deg;
  g.small_off = h->d_small_off;
  g.small_nbr = h->d_small_nbr;
  g.n = h->n;
  g.n_c = h->n_c;
  return g;
}

// ---- out-of-core streaming helpers --------------------------------------
// Stream words that positions [p, q) read (with the 4-word tail the 64-bit
// window may touch), from the host offsets.
void words_of(const lpa_handle *h, const uint64_t *offsets, uint64_t p, uint64_t q, uint64_t &w0, uint64_t &w1) {
  w0 = offsets[p] >> 5;
  w1 = std::min<uint64_t>(((offsets[q] + 31) >> 5) + 4, h->nwords + 4);
}

// Enqueues the copy of stream words [w0, w1) into buffer b on st and returns
// the buffer's virtual base: base[i] is stream word i for i in [w0, w1), and
// the base itself is 16-byte aligned.
const uint32_t *stage_words(lpa_handle *h, int b, uint64_t w0, uint64_t w1, cudaStream_t st) {
  const uint64_t sh = w0 & 3u;
  if (w1 - w0 + sh > h->wbuf_words) throw Fail{LPA_ERR_CAPACITY, "a stream range exceeds its buffer"};
  check(h, cudaMemcpyAsync(h->d_wbuf[b] + sh, h->h_wpinned + w0, (w1 - w0) * 4, cudaMemcpyHostToDevice, st),
        "stream range copy");
  h->streamed_bytes += (w1 - w0) * 4;
  h->wbuf_range[b] = -1;
  return reinterpret_cast<const uint32_t *>(reinterpret_cast<uintptr_t>(h->d_wbuf[b] + sh) - uintptr_t(w0) * 4);
}

// Buffer b's virtual base for stream words starting at w0 (as stage_words
// returns it), without copying.
const uint32_t *words_base(const lpa_handle *h, int b, uint64_t w0) {
  return reinterpret_cast<const uint32_t *>(reinterpret_cast<uintptr_t>(h->d_wbuf[b] + (w0 & 3u)) - uintptr_t(w0) * 4);
}

// The streamed scratch's virtual base for scratch indices [a0, ...): 16-byte
// aligned, so the count pass's bulk copies keep their alignment.
uint32_t *scratch_base(const lpa_handle *h, uint64_t a0) {
  return reinterpret_cast<uint32_t *>(reinterpret_cast<uintptr_t>(h->d_scratch + (a0 & 3u)) - uintptr_t(a0) * 4);
}

void cms_seeds(uint64_t seed, uint32_t out[kCmsDepth]) {
  // seed_r = low32(seed) ^ (0x9E3779B9 * (r + 1)), plus high32(seed) * 0x85EBCA6B
  const uint32_t lo = uint32_t(seed), hi = uint32_t(seed >> 32);
  for (int r = 0; r < kCmsDepth; r++) out[r] = (lo ^ (0x9E3779B9u * uint32_t(r + 1))) + hi * 0x85EBCA6Bu;
}

// Reads and clears the device error word.
lpa_status take_device_error(lpa_handle *h) {
  uint32_t err = 0;
  check(h, cudaMemcpyAsync(&err, h->d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream), "read error word");
  check(h, cudaStreamSynchronize(h->stream), "synchronize");
  if (err == kErrNone) return LPA_OK;
  check(h, cudaMemsetAsync(h->d_err, 0, sizeof(uint32_t), h->stream), "clear error word");
  switch (err) {
    case kErrBadStream:
      h->last_error = "bitstream decode left a vertex's bit range or produced an id >= n";
      return LPA_ERR_BAD_STREAM;
    case kErrCapacity:
      h->last_error = "a vertex exceeded its variant's planned capacity";
      return LPA_ERR_CAPACITY;
    case kErrTimeout:
      h->last_error = "a bounded device wait gave up";
      return LPA_ERR_TIMEOUT;
    default:
      h->last_error = "unknown device error";
      return LPA_ERR_CUDA;
  }
}

}  // namespace

namespace lpa_rt {

bool variant_capable(int v, const SegInfo &s, uint32_t cms_thr) {
  const bool any_cms = cms_thr != 0 && s.max_deg >= cms_thr;
  switch (v) {
    case LPA_VARIANT_PACKED:
      return !any_cms && s.max_deg <= kV2MaxDeg;
    case LPA_VARIANT_WARP:
      return !any_cms && s.max_deg <= kV1MaxDeg;
    case LPA_VARIANT_BLOCK:
    case LPA_VARIANT_TWO_PASS:
      return true;
    default:
      return false;
  }
}

// The reference's degree buckets: <16 packed warp, <128 warp, >=128 block
// (baselines/novaplus/novaplus_propogator.cuh:219-220, include/decoder.cuh:50-58).
int fixed_variant(const SegInfo &s) {
  switch (s.bucket) {
    case kTiny:
      return LPA_VARIANT_PACKED;
    case kMid:
      return LPA_VARIANT_WARP;
    default:
      return LPA_VARIANT_BLOCK;
  }
}

}  // namespace lpa_rt

// ------------------------------------------------------------------ plan ---
std::vector<SegInfo> lpa_rt::make_segments(const uint32_t *deg, uint64_t n, uint64_t n_c, uint32_t cms) {
  std::vector<SegInfo> segs;
  auto bucket_of = [&](uint32_t d) -> uint8_t {
    if ((cms != 0 && d >= cms) || d > kV1MaxDeg) return kHeavy;
    if (d < 16) return kTiny;
    if (d < 128) return kMid;
    return kLarge;
  };
  SegInfo cur{};
  bool open = false;
  auto close = [&]() {
    if (open) segs.push_back(cur);
    open = false;
  };
  for (uint64_t p = 0; p < n; p++) {
    const uint32_t d = deg[p];
    const uint8_t region = p < n_c ? 0 : 1;
    if (d == 0) {
      // isolated vertices need no work; they only end a segment
      close();
      continue;
    }
    const uint8_t b = bucket_of(d);
    if (open && (cur.bucket != b || cur.region != region || cur.end - cur.begin >= kSegPositions[b] ||
                 cur.arcs + d > kSegArcs)) {
      close();
    }
    if (!open) {
      cur = SegInfo{uint32_t(p), uint32_t(p), b, region, 0, 0, 0, 0};
      open = true;
    }
    cur.end = uint32_t(p + 1);
    cur.max_deg = std::max(cur.max_deg, d);
    cur.arcs += d;
  }
  close();
  return segs;
}

static void build_segments(lpa_handle *h) {
  h->segs = make_segments(h->h_deg.data(), h->n, h->n_c, h->opts.cms_threshold);
}

// The plan's work lists, built on the device (plan.cu): a plan change costs a
// few launches and one copy of the list sizes, not a host loop over n.
static void upload_range_lists(lpa_handle *h);

// The block path's sketch hubs keep their labels between the sketch's two
// passes in a per-block spill area (at most 2 GiB in all; larger hubs decode
// twice), allocated once a plan gives k_iterate heavy items.
static void ensure_hub_spill(lpa_handle *h) {
  if (h->d_hub_spill || h->n_heavy == 0 || h->max_sketch_deg == 0) return;
  const uint64_t per_block = std::min<uint64_t>(h->max_sketch_deg, (2ull << 30) / 4 / uint64_t(std::max(1, h->grid)));
  h->d_hub_spill = dalloc<uint32_t>(h, per_block * uint64_t(h->grid), "hub spill");
  h->hub_spill_words = uint32_t(per_block);
}

static void upload_lists(lpa_handle *h) {
  h2d(h, h->d_seg_var, h->variant.data(), h->variant.size(), "upload variants");
  if (h->streamed) {
    upload_range_lists(h);
    return;
  }
  PlanInputs in{};
  in.segs = h->d_segdev;
  in.seg_begin = 0;
  in.nseg = uint32_t(h->segs.size());
  in.c_begin = 0;
  in.c_end = h->n_c;
  in.s_begin = h->n_c;
  in.s_end = h->n;
  in.var = h->d_seg_var;
  in.deg = h->d_deg;
  in.vertices = h->d_vertices;
  in.pidx = h->d_pidx;
  in.arc_off = h->d_arc_off;
  in.offsets = h->d_offsets;
  in.small_off = h->d_small_off;
  in.words = h->d_words;
  in.small_nbr = h->d_small_nbr;
  in.scratch = h->d_scratch;
  in.n = h->n;
  in.n_c = h->n_c;
  in.cms = h->opts.cms_threshold;
  in.wmax = h->tune.warp_max_degree;
  in.warp_positions = h->tune.warp_positions;
  in.group_positions = h->tune.group_positions;
  in.num_sms = h->num_sms;
  auto regrow = [&](auto *&ptr, size_t &cap, size_t need, const char *what) {
    if (need <= cap && ptr) return;
    if (ptr) {
      auto it = std::find(h->allocations.begin(), h->allocations.end(), (void *)ptr);
      if (it != h->allocations.end()) h->allocations.erase(it);
      cudaFree(ptr);
    }
    cap = need + need / 4 + 16;
    ptr = dalloc<std::remove_reference_t<decltype(*ptr)>>(h, cap, what);
  };
  PlanOutputs out{};
  out.grow = [&](PlanOutputs &o) -> cudaError_t {
    regrow(h->d_items, h->items_cap, size_t(o.n_heavy) + o.n_light, "work items");
    regrow(h->d_groups, h->groups_cap, o.n_groups, "decode groups");
    regrow(h->d_citems, h->citems_cap, o.n_cwarp, "count items");
    regrow(h->d_cblock, h->cblock_cap, o.n_cblock, "count block items");
    regrow(h->d_packed, h->packed_cap, o.n_packed, "packed chunks");
    o.items = h->d_items;
    o.groups = h->d_groups;
    o.cwarp = h->d_citems;
    o.cblock = h->d_cblock;
    o.packed = h->d_packed;
    return cudaSuccess;
  };
  std::string where;
  const cudaError_t e = h->plan_builder.build(in, out, h->stream, where);
  check(h, e, ("build work lists: " + where).c_str());
  check(h, cudaStreamSynchronize(h->stream), "build work lists");
  h->n_heavy = out.n_heavy;
  h->n_light = out.n_light;
  h->n_packed = out.n_packed;
  h->n_groups = out.n_groups;
  h->n_cblock = out.n_cblock;
  h->n_cwarp = out.n_cwarp;
  ensure_hub_spill(h);
  h->plan_version++;
  // the resident blocks (the warps take decode groups from a work queue),
  // fewer when there are fewer groups than warps
  h->grid_decode = int(std::max<uint64_t>(
      1, std::min<uint64_t>((uint64_t(h->n_groups) + kWarps - 1) / kWarps, uint64_t(h->num_sms) * h->occ_decode)));
}

// The work lists of every range of a streamed handle, each built by the
// device builder over the range's segments and positions.
static void upload_range_lists(lpa_handle *h) {
  auto regrow = [&](auto *&ptr, size_t &cap, size_t need, const char *what) {
    if (need <= cap && ptr) return;
    if (ptr) {
      auto it = std::find(h->allocations.begin(), h->allocations.end(), (void *)ptr);
      if (it != h->allocations.end()) h->allocations.erase(it);
      cudaFree(ptr);
    }
    cap = need + need / 4 + 16;
    ptr = dalloc<std::remove_reference_t<decltype(*ptr)>>(h, cap, what);
  };
  h->n_heavy = h->n_light = h->n_packed = h->n_groups = h->n_cblock = h->n_cwarp = 0;
  for (size_t k = 0; k < h->ranges.size(); k++) {
    StreamRange &r = h->ranges[k];
    PlanInputs in{};
    in.segs = h->d_segdev;
    in.seg_begin = r.s0;
    in.nseg = r.s1 - r.s0;
    in.c_begin = r.p0;
    in.c_end = r.p1;
    in.s_begin = r.last ? h->n_c : h->n;
    in.s_end = h->n;
    in.var = h->d_seg_var;
    in.deg = h->d_deg;
    in.vertices = h->d_vertices;
    in.pidx = h->d_pidx;
    in.arc_off = h->d_arc_off;
    in.offsets = h->d_offsets;
    in.small_off = h->d_small_off;
    in.words = words_base(h, int(k & 1), r.w0);  // prefetch ranges point into the range's buffer
    in.small_nbr = h->d_small_nbr;
    in.scratch = h->d_scratch ? scratch_base(h, r.a0) : nullptr;
    in.n = h->n;
    in.n_c = h->n_c;
    in.cms = h->opts.cms_threshold;
    in.wmax = h->tune.warp_max_degree;
    in.warp_positions = h->tune.warp_positions;
    in.group_positions = h->tune.group_positions;
    in.num_sms = h->num_sms;
    PlanOutputs out{};
    out.grow = [&](PlanOutputs &o) -> cudaError_t {
      regrow(r.items, r.items_cap, size_t(o.n_heavy) + o.n_light, "range work items");
      regrow(r.groups, r.groups_cap, o.n_groups, "range decode groups");
      regrow(r.cwarp, r.cwarp_cap, o.n_cwarp, "range count items");
      regrow(r.cblock, r.cblock_cap, o.n_cblock, "range count block items");
      regrow(r.packed, r.packed_cap, o.n_packed, "range packed chunks");
      o.items = r.items;
      o.groups = r.groups;
      o.cwarp = r.cwarp;
      o.cblock = r.cblock;
      o.packed = r.packed;
      return cudaSuccess;
    };
    std::string where;
    const cudaError_t e = h->plan_builder.build(in, out, h->stream, where);
    check(h, e, ("build range work lists: " + where).c_str());
    check(h, cudaStreamSynchronize(h->stream), "build range work lists");
    r.n_heavy = out.n_heavy;
    r.n_light = out.n_light;
    r.n_packed = out.n_packed;
    r.n_groups = out.n_groups;
    r.n_cblock = out.n_cblock;
    r.n_cwarp = out.n_cwarp;
    r.grid_decode = int(std::max<uint64_t>(
        1, std::min<uint64_t>((uint64_t(r.n_groups) + kWarps - 1) / kWarps, uint64_t(h->num_sms) * h->occ_decode)));
    h->n_heavy += r.n_heavy;
    h->n_light += r.n_light;
    h->n_packed += r.n_packed;
    h->n_groups += r.n_groups;
    h->n_cblock += r.n_cblock;
    h->n_cwarp += r.n_cwarp;
  }
  ensure_hub_spill(h);
  h->plan_version++;
}

static void ensure_two_pass_scratch(lpa_handle *h) {
  if (h->d_scratch) return;
  std::vector<uint64_t> &off = h->h_arc_off;
  off.assign(h->n + 1, 0);
  for (uint64_t p = 0; p < h->n; p++) off[p + 1] = off[p] + h->h_deg[p];
  h->d_arc_off = dalloc<uint64_t>(h, h->n + 1, "arc offsets");
  h2d(h, h->d_arc_off, off.data(), h->n + 1, "upload arc offsets");
  // + 4: a 16-byte-aligned bulk copy may read up to 12 bytes past the last label
  // (streamed: one range's labels at a time, after up to 3 words of alignment)
  h->d_scratch = dalloc<uint32_t>(h, h->streamed ? h->scratch_words : off[h->n_c] + 4, "two-pass scratch");
  // where every compressed position's segments start, for the pre-pass
  const uint64_t nc = std::max<uint64_t>(1, h->n_c);
  h->d_pidx = dalloc<uint4>(h, nc, "position index");
  h->d_cursor = dalloc<uint32_t>(h, nc, "pre-pass cursors");
  check(h, cudaMemsetAsync(h->d_cursor, 0, nc * sizeof(uint32_t), h->stream), "clear cursors");
  if (h->streamed) {
    for (const StreamRange &r : h->ranges) {
      if (r.p1 <= r.p0) continue;
      DevGraph g = dev_graph(h);
      g.words = stage_words(h, 0, r.w0, r.w1, h->stream);
      const int blocks = int(std::min<uint64_t>((r.p1 - r.p0 + 127) / 128, uint64_t(h->num_sms) * 32));
      k_pos_index<<<std::max(blocks, 1), 128, 0, h->stream>>>(g, h->d_pidx, h->d_err, r.p0, r.p1);
      check(h, cudaGetLastError(), "position index launch");
      check(h, cudaStreamSynchronize(h->stream), "position index");  // the buffer is reused by the next range
    }
  } else if (h->n_c) {
    const int blocks = int(std::min<uint64_t>((h->n_c + 127) / 128, uint64_t(h->num_sms) * 32));
    k_pos_index<<<std::max(blocks, 1), 128, 0, h->stream>>>(dev_graph(h), h->d_pidx, h->d_err, 0, h->n_c);
    check(h, cudaGetLastError(), "position index launch");
  }
  lpa_status st = take_device_error(h);
  if (st != LPA_OK) throw Fail{st, "position index: " + h->last_error};
  check(h, cudaStreamSynchronize(h->stream), "arc offsets");
}

static void apply_dispatch(lpa_handle *h, int dispatch, int force) {
  h->variant.resize(h->segs.size());
  bool any_two = false;
  for (size_t s = 0; s < h->segs.size(); s++) {
    int v = h->fixed[s];
    if (dispatch == LPA_DISPATCH_FORCE && variant_capable(force, h->segs[s], h->opts.cms_threshold)) v = force;
    h->variant[s] = uint8_t(v);
    any_two |= v == LPA_VARIANT_TWO_PASS;
  }
  if (any_two) ensure_two_pass_scratch(h);
  upload_lists(h);
}

// Ranges of a streamed handle: consecutive plan segments of the compressed
// region whose stream fits one buffer and whose labels fit the scratch; the
// small CSR's segments go with the last range (they read no stream).
static void build_ranges(lpa_handle *h) {
  const uint64_t *off = h->create_offsets;
  std::vector<uint64_t> arc(h->n_c + 1, 0);
  for (uint64_t p = 0; p < h->n_c; p++) arc[p + 1] = arc[p] + h->h_deg[p];
  auto fits = [&](uint64_t p0, uint64_t p1) {
    uint64_t w0, w1;
    words_of(h, off, p0, p1, w0, w1);
    return w1 - w0 + 3 <= h->wbuf_words && arc[p1] - arc[p0] + 8 <= h->scratch_words;
  };
  h->ranges.clear();
  const uint32_t S = uint32_t(h->segs.size());
  uint32_t s = 0;
  StreamRange cur;
  while (s < S && h->segs[s].region == 0) {
    const SegInfo &sg = h->segs[s];
    if (!fits(sg.begin, sg.end))
      throw Fail{LPA_ERR_CAPACITY, "a segment's stream or labels exceed the stream budget"};
    if (s > cur.s0 && !fits(cur.p0, sg.end)) {
      cur.p1 = sg.begin;
      cur.s1 = s;
      h->ranges.push_back(cur);
      cur = StreamRange{};
      cur.p0 = sg.begin;
      cur.s0 = s;
    }
    s++;
  }
  cur.p1 = h->n_c;
  cur.s1 = S;  // the small CSR's segments too
  cur.last = true;
  h->ranges.push_back(cur);
  // every range takes one block of work-queue counters per iteration
  if (h->ranges.size() > size_t(kMaxRunSlots))
    throw Fail{LPA_ERR_CAPACITY, "stream budget too small: more ranges than work-counter slots"};
  for (StreamRange &r : h->ranges) {
    words_of(h, off, r.p0, std::max(r.p1, r.p0), r.w0, r.w1);
    r.a0 = arc[r.p0];
    r.a1 = arc[r.p1];
  }
}

static void build_plan(lpa_handle *h) {
  // degrees, decoded once on the device (validates the stream as well)
  h->d_deg = dalloc<uint32_t>(h, h->n, "degrees");
  uint32_t *d_itv = nullptr;
  check(h, cudaMalloc(&d_itv, std::max<uint64_t>(1, h->n) * sizeof(uint32_t)), "interval counts");
  const int threads = 128;
  auto degree_pass = [&](const DevGraph &g, uint64_t p0, uint64_t p1) {
    if (p1 <= p0) return;
    const int blocks = int(std::min<uint64_t>((p1 - p0 + threads - 1) / threads, uint64_t(h->num_sms) * 32));
    k_degree_count<<<std::max(blocks, 1), threads, 0, h->stream>>>(g, h->d_deg, d_itv, h->d_err, p0, p1);
    check(h, cudaGetLastError(), "degree kernel launch");
  };
  if (h->streamed) {
    // compressed positions in chunks whose stream fits one buffer, then the small CSR
    const uint64_t *off = h->create_offsets;
    uint64_t p = 0;
    while (p < h->n_c) {
      uint64_t q = p + 1, w0, w1;
      words_of(h, off, p, q, w0, w1);
      if (w1 - w0 + 3 > h->wbuf_words) throw Fail{LPA_ERR_CAPACITY, "a vertex's stream exceeds the stream budget"};
      uint64_t step = 1;
      while (q < h->n_c) {  // grow the chunk by doubling steps, then halving
        const uint64_t t = std::min<uint64_t>(h->n_c, q + step);
        words_of(h, off, p, t, w0, w1);
        if (w1 - w0 + 3 <= h->wbuf_words) {
          q = t;
          step *= 2;
        } else if (step > 1) {
          step /= 2;
        } else {
          break;
        }
      }
      words_of(h, off, p, q, w0, w1);
      DevGraph g = dev_graph(h);
      g.words = stage_words(h, 0, w0, w1, h->stream);
      degree_pass(g, p, q);
      check(h, cudaStreamSynchronize(h->stream), "degree pass");  // the buffer is reused by the next chunk
      p = q;
    }
    degree_pass(dev_graph(h), h->n_c, h->n);
  } else {
    degree_pass(dev_graph(h), 0, h->n);
  }
  lpa_status st = take_device_error(h);
  if (st != LPA_OK) throw Fail{st, "degree pass: " + h->last_error};
  h->h_deg.resize(h->n);
  check(h, cudaMemcpy(h->h_deg.data(), h->d_deg, h->n * sizeof(uint32_t), cudaMemcpyDeviceToHost),
        "read degrees");
  std::vector<uint32_t> itv(h->n);
  check(h, cudaMemcpy(itv.data(), d_itv, h->n * sizeof(uint32_t), cudaMemcpyDeviceToHost), "read interval counts");
  cudaFree(d_itv);
  h->m = 0;
  h->max_deg = 0;
  for (uint64_t p = 0; p < h->n; p++) {
    h->m += h->h_deg[p];
    h->max_deg = std::max<uint64_t>(h->max_deg, h->h_deg[p]);
  }
  build_segments(h);
  for (auto &sg : h->segs) {
    uint64_t iv = 0;
    for (uint32_t p = sg.begin; p < sg.end; p++) iv += itv[p];
    sg.intervals = uint32_t(std::min<uint64_t>(iv, 0xFFFFFFFFull));
  }
  if (h->streamed) build_ranges(h);
  h->fixed.resize(h->segs.size());
  for (size_t s = 0; s < h->segs.size(); s++) h->fixed[s] = uint8_t(fixed_variant(h->segs[s]));
  std::vector<Seg> ds(h->segs.size());
  for (size_t s = 0; s < h->segs.size(); s++) ds[s] = Seg{h->segs[s].begin, h->segs[s].end};
  h->d_segs = dalloc<Seg>(h, ds.size(), "segments");
  h->d_seg_var = dalloc<uint8_t>(h, ds.size(), "segment variants");
  h->d_seg_changed = dalloc<uint32_t>(h, ds.size(), "segment changed counts");
  h->d_seg_changed_prev = dalloc<uint32_t>(h, ds.size(), "segment changed counts");
  check(h, cudaMemsetAsync(h->d_seg_changed, 0, std::max<size_t>(1, ds.size()) * sizeof(uint32_t), h->stream),
        "clear segment counts");
  check(h, cudaMemsetAsync(h->d_seg_changed_prev, 0, std::max<size_t>(1, ds.size()) * sizeof(uint32_t), h->stream),
        "clear segment counts");
  h2d(h, h->d_segs, ds.data(), ds.size(), "upload segments");
  std::vector<SegDev> sd(h->segs.size());
  for (size_t s = 0; s < h->segs.size(); s++) {
    const SegInfo &si = h->segs[s];
    sd[s] = SegDev{si.begin, si.end, si.max_deg, si.bucket, si.region, 0, 0, si.arcs};
  }
  h->d_segdev = dalloc<SegDev>(h, sd.size(), "segment table");
  h2d(h, h->d_segdev, sd.data(), sd.size(), "upload segment table");
  check(h, cudaStreamSynchronize(h->stream), "upload segments");
  h->d_seg_cycles = dalloc<long long>(h, h->segs.size(), "segment cycles");
  h->d_ktime = dalloc<unsigned long long>(h, 2 * kBusyKernels, "kernel busy spans");
  check(h, cudaMemsetAsync(h->d_seg_cycles, 0, std::max<size_t>(1, h->segs.size()) * sizeof(long long), h->stream),
        "clear cycles");

  // global exact-count tables for exact vertices above the shared table
  uint64_t big = 0;
  for (uint64_t p = 0; p < h->n; p++) {
    const uint32_t d = h->h_deg[p];
    const bool cms = h->opts.cms_threshold != 0 && d >= h->opts.cms_threshold;
    if (!cms && d > kBlockMaxSmemDeg) big = std::max<uint64_t>(big, d);
    if (cms) h->max_sketch_deg = std::max(h->max_sketch_deg, d);
  }
  if (big) {
    h->gtab_slots = next_pow2_host(2 * big);
    const uint64_t per_block = uint64_t(h->gtab_slots) * 2 * sizeof(uint32_t);
    // one table per block of the persistent kernel; at most 2 GiB of tables
    h->gtab_blocks = int(std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(h->grid), (2ull << 30) / per_block)));
    h->grid = std::min(h->grid, h->gtab_blocks);
    h->d_gtab = dalloc<uint32_t>(h, uint64_t(h->gtab_blocks) * 2 * h->gtab_slots, "global count tables");
    check(h, cudaMemsetAsync(h->d_gtab, 0, uint64_t(h->gtab_blocks) * per_block, h->stream), "clear tables");
  }
  apply_dispatch(h, h->opts.dispatch == LPA_DISPATCH_FORCE ? LPA_DISPATCH_FORCE : LPA_DISPATCH_FIXED,
                 h->opts.force_variant);
}

static IterArgs iter_args(lpa_handle *h, unsigned long long *changed, uint32_t *work) {
  IterArgs a{};
  a.g = dev_graph(h);
  a.labs0 = h->d_lab[0];
  a.labs1 = h->d_lab[1];
  a.parity0 = uint32_t(h->cur);
  a.it_dev = h->loop_it;
  a.changed = changed;
  a.work = work;
  a.err = h->d_err;
  a.segs = h->d_segs;
  a.seg_var = h->d_seg_var;
  a.heavy = h->d_items;
  a.n_heavy = h->n_heavy;
  a.light = h->d_items + h->n_heavy;
  a.n_light = h->n_light;
  a.groups = h->d_groups;
  a.n_groups = h->n_groups;
  a.cblock = h->d_cblock;
  a.n_cblock = h->n_cblock;
  a.cwarp = h->d_citems;
  a.n_cwarp = h->n_cwarp;
  a.warp_claim = h->tune.warp_claim;
  a.packed = h->d_packed;
  a.n_packed = h->n_packed;
  a.cw_packed = h->cw_packed;
  a.pidx = h->d_pidx;
  a.cursor = h->d_cursor;
  a.seg_cycles = (h->opts.record_timings >= 2 || h->collect_cycles) ? h->d_seg_cycles : nullptr;
  a.cw_iterate = h->cw_iterate;
  a.cw_decode = h->cw_decode;
  a.cw_count = h->cw_count;
  a.ktime = (h->collect_cycles || h->measure_busy || h->learner_spans) ? h->d_ktime : nullptr;
  a.seg_changed = h->learner ? h->d_seg_changed : nullptr;
  a.cms_thr = h->opts.cms_threshold;
  for (int r = 0; r < kCmsDepth; r++) a.seeds[r] = h->seeds[r];
  a.scratch = h->d_scratch;
  a.arc_off = h->d_arc_off;
  a.scratch_labels = 1;
  a.gtab = h->d_gtab;
  a.gtab_slots = h->gtab_slots;
  a.gbase = h->d_gbase;
  a.n_gbase = h->d_gbase ? h->n_graphs : 0u;
  a.wend = (h->nwords + 4) & ~uint64_t(3);
  a.hub_spill = h->d_hub_spill;
  a.hub_spill_words = h->hub_spill_words;
  return a;
}

// Enqueues one iteration (no host synchronisation).  Swaps the buffers.  The
// changed counter and the two queue counters of the iteration's slot must be
// zero.
static void enqueue_streamed_iteration(lpa_handle *h, unsigned long long *changed, uint32_t *work);

static void enqueue_iteration(lpa_handle *h, unsigned long long *changed, uint32_t *work) {
  if (h->streamed) {
    enqueue_streamed_iteration(h, changed, work);
    return;
  }
  const bool timed = h->opts.record_timings && h->events_ready;
  const IterArgs a = iter_args(h, changed, work);
  // events only around the kernels that run: an event costs a few us of
  // device time, which small graphs would otherwise count
  int ne = 0;
  auto mark = [&](int kernel) {
    if (!timed) return;
    h->ev_kernel[ne] = kernel;
    cudaEventRecord(h->ev[ne++], h->stream);
  };
  mark(-1);
  if (h->n_groups) {
    launch_decode_two_pass(h->tune.gather_cache, h->tune.stage_stream, h->grid_decode, h->stream, a);
    h->launches++;
    mark(0);
  }
  if (h->n_cblock + h->n_cwarp) {
    launch_count_two_pass(h->tune.bulk_stage != 0, h->grid_count, h->stream, a);
    h->launches++;
    mark(1);
  }
  if (h->n_packed) {
    k_packed<<<h->grid_packed, kThreads, 0, h->stream>>>(a);
    h->launches++;
    mark(2);
  }
  if (h->n_heavy + h->n_light) {
    k_iterate<<<h->grid, kThreads, kSmemBytes, h->stream>>>(a);
    h->launches++;
    mark(3);
  }
  if (h->d_gtrack) {
    lpa_rt_enqueue_track(h);
    h->launches += 2;
  }
  h->ev_used = ne;
  h->cur ^= 1;
}

// One iteration of a streamed handle: range by range, each range's stream
// words copied on the copy stream into one of two buffers (the copy of range
// k + 1 overlaps the kernels of range k), its kernels then launched on the
// handle's stream over its own work lists with the buffer's and the scratch's
// virtual bases.  A buffer that still holds its range's words (two ranges or
// fewer) is not copied again.  Every range reads the same label buffer and
// writes the other; the buffers swap once, after the last range.
static void enqueue_streamed_iteration(lpa_handle *h, unsigned long long *changed, uint32_t *work) {
  const bool timed = h->opts.record_timings && h->events_ready;
  if (timed) {
    h->ev_kernel[0] = -1;
    cudaEventRecord(h->ev[0], h->stream);
  }
  const size_t R = h->ranges.size();
  std::vector<const uint32_t *> base(R, nullptr);
  auto issue_copy = [&](size_t k) {
    const StreamRange &r = h->ranges[k];
    const int b = int(k & 1);
    if (h->wbuf_range[b] == int(k)) {
      base[k] = words_base(h, b, r.w0);
      return;
    }
    check(h, cudaStreamWaitEvent(h->copy_stream, h->ev_free[b], 0), "wait for a free stream buffer");
    base[k] = stage_words(h, b, r.w0, r.w1, h->copy_stream);
    check(h, cudaEventRecord(h->ev_ready[b], h->copy_stream), "stream buffer ready");
    h->wbuf_range[b] = int(k);
  };
  if (R) issue_copy(0);
  for (size_t k = 0; k < R; k++) {
    if (k + 1 < R) issue_copy(k + 1);
    const StreamRange &r = h->ranges[k];
    const int b = int(k & 1);
    check(h, cudaStreamWaitEvent(h->stream, h->ev_ready[b], 0), "wait for the stream range");
    IterArgs a = iter_args(h, changed, work + kWorkCounters * k);
    a.g.words = base[k];
    a.heavy = r.items;
    a.n_heavy = r.n_heavy;
    a.light = r.items + r.n_heavy;
    a.n_light = r.n_light;
    a.groups = r.groups;
    a.n_groups = r.n_groups;
    a.cblock = r.cblock;
    a.n_cblock = r.n_cblock;
    a.cwarp = r.cwarp;
    a.n_cwarp = r.n_cwarp;
    a.packed = r.packed;
    a.n_packed = r.n_packed;
    a.scratch = h->d_scratch ? scratch_base(h, r.a0) : nullptr;
    a.wend = r.w1 & ~uint64_t(3);
    if (r.n_groups) {
      launch_decode_two_pass(h->tune.gather_cache, h->tune.stage_stream, r.grid_decode, h->stream, a);
      h->launches++;
    }
    if (r.n_cblock + r.n_cwarp) {
      launch_count_two_pass(h->tune.bulk_stage != 0, h->grid_count, h->stream, a);
      h->launches++;
    }
    if (r.n_packed) {
      k_packed<<<h->grid_packed, kThreads, 0, h->stream>>>(a);
      h->launches++;
    }
    if (r.n_heavy + r.n_light) {
      k_iterate<<<h->grid, kThreads, kSmemBytes, h->stream>>>(a);
      h->launches++;
    }
    check(h, cudaEventRecord(h->ev_free[b], h->stream), "stream buffer free");
  }
  if (h->d_gtrack) {
    lpa_rt_enqueue_track(h);
    h->launches += 2;
  }
  if (timed) {
    h->ev_kernel[1] = -1;  // the whole iteration: no per-kernel split
    cudaEventRecord(h->ev[1], h->stream);
    h->ev_used = 2;
  } else {
    h->ev_used = 0;
  }
  h->cur ^= 1;
}

static void collect_times(lpa_handle *h) {
  if (!(h->opts.record_timings && h->events_ready)) return;
  auto ms = [&](int a, int b) {
    float t = 0;
    if (cudaEventElapsedTime(&t, h->ev[a], h->ev[b]) != cudaSuccess) {
      cudaGetLastError();
      return 0.0;
    }
    return double(t);
  };
  for (int v = 0; v < 4; v++) h->variant_ms[v] = 0;
  double k_ms[4] = {0, 0, 0, 0};  // pre-pass, count pass, k_packed, k_iterate
  for (int e = 1; e < h->ev_used; e++)
    if (h->ev_kernel[e] >= 0 && h->ev_kernel[e] < 4) k_ms[h->ev_kernel[e]] = ms(e - 1, e);
  h->decode_ms = k_ms[0];
  h->count_ms = k_ms[1];
  h->packed_ms = k_ms[2];
  h->iterate_ms = k_ms[3];
  h->last_iter_ms = h->ev_used > 1 ? ms(0, h->ev_used - 1) : 0.0;
}

// ------------------------------------------------------------------ C ABI --
extern "C" {

const char *lpa_status_str(lpa_status s) {
  switch (s) {
    case LPA_OK: return "ok";
    case LPA_ERR_CUDA: return "CUDA error";
    case LPA_ERR_OOM: return "out of device memory";
    case LPA_ERR_BAD_STREAM: return "malformed bitstream";
    case LPA_ERR_TIMEOUT: return "device wait timed out";
    case LPA_ERR_INVALID_ARG: return "invalid argument";
    case LPA_ERR_IO: return "file missing or malformed";
    case LPA_ERR_NO_DEVICE: return "no CUDA device";
    case LPA_ERR_CAPACITY: return "planned capacity exceeded";
  }
  return "unknown status";
}

const char *lpa_version(void) { return "lpa_b200 0.1 (sm_100a)"; }

void lpa_opts_default(lpa_opts *o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->device = 0;
  o->cms_threshold = 0;
  o->cms_seed = 1;
  o->dispatch = LPA_DISPATCH_FIXED;
  o->force_variant = LPA_VARIANT_BLOCK;
  o->stream = nullptr;
  o->record_timings = 0;
  o->verbose = 0;
}

lpa_status lpa_create(const lpa_graph_desc *g, const lpa_opts *o, lpa_handle **out) {
  if (!g || !out) return LPA_ERR_INVALID_ARG;
  *out = nullptr;
  const uint64_t n = g->num_vertices, n_c = g->num_compressed;
  if (n == 0 || n > 0xFFFFFFFEull || n_c > n || !g->vertices) return LPA_ERR_INVALID_ARG;
  if (n_c > 0 && (!g->words || !g->offsets)) return LPA_ERR_INVALID_ARG;
  if (n > n_c && !g->small_offset) return LPA_ERR_INVALID_ARG;
  if (g->num_small_arcs > 0 && !g->small_graph) return LPA_ERR_INVALID_ARG;
  // host-side format checks: monotone offsets inside the stream, small CSR sizes
  if (n_c > 0) {
    if (g->offsets[0] != 0) return LPA_ERR_BAD_STREAM;
    for (uint64_t i = 0; i < n_c; i++)
      if (g->offsets[i + 1] < g->offsets[i]) return LPA_ERR_BAD_STREAM;
    if ((g->offsets[n_c] + 31) / 32 > g->num_words) return LPA_ERR_BAD_STREAM;
  }
  if (n > n_c) {
    if (g->small_offset[0] != 0 || g->small_offset[n - n_c] != g->num_small_arcs) return LPA_ERR_INVALID_ARG;
    for (uint64_t i = 0; i < n - n_c; i++)
      if (g->small_offset[i + 1] < g->small_offset[i]) return LPA_ERR_INVALID_ARG;
  }

  lpa_handle *h = new (std::nothrow) lpa_handle();
  if (!h) return LPA_ERR_OOM;
  if (o) h->opts = *o;
  else lpa_opts_default(&h->opts);
  if (h->opts.dispatch == LPA_DISPATCH_LEARNED && h->opts.record_timings < 1) h->opts.record_timings = 1;
  try {
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      delete h;
      return LPA_ERR_NO_DEVICE;
    }
    if (h->opts.device < 0 || h->opts.device >= count) throw Fail{LPA_ERR_INVALID_ARG, "device ordinal"};
    h->device = h->opts.device;
    check(h, cudaSetDevice(h->device), "cudaSetDevice");
    check(h, cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device), "SM count");
    if (h->opts.stream) {
      h->stream = static_cast<cudaStream_t>(h->opts.stream);
    } else {
      check(h, cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "stream");
      h->own_stream = true;
    }
    check(h, cudaFuncSetAttribute(k_iterate, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes)),
          "smem attr");
    check(h, prepare_decode_two_pass(), "smem attr");
    check(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&h->occ, k_iterate, kThreads, kSmemBytes), "occupancy");
    h->occ = std::max(1, h->occ);
    h->grid = h->num_sms * h->occ;
    int occ_count = 1;  // one grid for both forms
    check(h, occupancy_count_two_pass(&occ_count), "occupancy");
    h->grid_count = h->num_sms * std::max(1, occ_count);
    int occ_decode = 1;  // one grid for every form
    check(h, occupancy_decode_two_pass(&occ_decode), "occupancy");
    h->occ_decode = std::max(1, occ_decode);
    // 960 is divisible by every resident warp count these kernels reach (16..64 in steps of 8)
    const auto weight = [](int blocks) { return uint32_t(std::max(1, 960 / (std::max(1, blocks) * kWarps))); };
    h->cw_iterate = weight(h->occ);
    h->cw_count = weight(occ_count);
    h->cw_decode = weight(occ_decode);
    int occ_packed = 1;
    check(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_packed, k_packed, kThreads, 0), "occupancy");
    h->grid_packed = h->num_sms * std::max(1, occ_packed);
    h->cw_packed = weight(occ_packed);

    h->n = n;
    h->n_c = n_c;
    h->nwords = g->num_words;
    h->m_small = g->num_small_arcs;
    h->total_bits = n_c ? g->offsets[n_c] : 0;
    cms_seeds(h->opts.cms_seed, h->seeds);

    // device copies; the stream gets 4 zero words of tail for the 64-bit window
    const uint64_t wcount = h->nwords + 4;
    h->streamed = h->opts.stream_budget != 0 && n_c != 0;
    if (h->streamed) {
      // out of core: the stream in pinned host memory, two device buffers of
      // a quarter of the budget each, the label scratch in the other half
      h->wbuf_words = h->opts.stream_budget / 16;
      h->scratch_words = h->opts.stream_budget / 8;
      if (h->wbuf_words < 64 || h->scratch_words < 64) throw Fail{LPA_ERR_INVALID_ARG, "stream budget too small"};
      check(h, cudaMallocHost(&h->h_wpinned, wcount * sizeof(uint32_t)), "pinned stream");
      std::memcpy(h->h_wpinned, g->words, h->nwords * sizeof(uint32_t));
      std::memset(h->h_wpinned + h->nwords, 0, 4 * sizeof(uint32_t));
      for (int b = 0; b < 2; b++) h->d_wbuf[b] = dalloc<uint32_t>(h, h->wbuf_words, "stream buffer");
      check(h, cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking), "copy stream");
      for (int b = 0; b < 2; b++) {
        check(h, cudaEventCreateWithFlags(&h->ev_ready[b], cudaEventDisableTiming), "events");
        check(h, cudaEventCreateWithFlags(&h->ev_free[b], cudaEventDisableTiming), "events");
      }
    } else {
      h->d_words = dalloc<uint32_t>(h, wcount, "bitstream");
      check(h, cudaMemsetAsync(h->d_words, 0, wcount * sizeof(uint32_t), h->stream), "clear bitstream");
      h2d(h, h->d_words, g->words, h->nwords, "upload bitstream");
    }
    h->d_offsets = dalloc<uint64_t>(h, n_c + 1, "offsets");
    if (n_c) h2d(h, h->d_offsets, g->offsets, n_c + 1, "upload offsets");
    h->d_vertices = dalloc<uint32_t>(h, n, "vertices");
    h2d(h, h->d_vertices, g->vertices, n, "upload vertices");
    h->d_small_off = dalloc<uint32_t>(h, n - n_c + 1, "small offsets");
    if (n > n_c) h2d(h, h->d_small_off, g->small_offset, n - n_c + 1, "upload small offsets");
    h->d_small_nbr = dalloc<uint32_t>(h, h->m_small, "small neighbours");
    h2d(h, h->d_small_nbr, g->small_graph, h->m_small, "upload small neighbours");
    h->d_lab[0] = dalloc<uint32_t>(h, n, "labels");
    h->d_lab[1] = dalloc<uint32_t>(h, n, "labels");
    h->changed_slots = kMaxRunSlots;
    h->d_changed = dalloc<unsigned long long>(h, h->changed_slots, "changed counters");
    h->d_work = dalloc<uint32_t>(h, kWorkCounters * size_t(h->changed_slots), "work counters");
    check(h, cudaMemsetAsync(h->d_work, 0, kWorkCounters * size_t(h->changed_slots) * sizeof(uint32_t), h->stream),
          "clear work counters");
    check(h, cudaMemsetAsync(h->d_changed, 0, h->changed_slots * sizeof(unsigned long long), h->stream),
          "clear counters");
    h->d_err = dalloc<uint32_t>(h, 1, "error word");
    check(h, cudaMemsetAsync(h->d_err, 0, sizeof(uint32_t), h->stream), "clear error word");
    check(h, cudaMallocHost(&h->h_pinned, sizeof(unsigned long long) * 64), "pinned readback");
    for (auto &e : h->ev) check(h, cudaEventCreate(&e), "events");
    h->events_ready = true;

    h->create_offsets = g->offsets;
    build_plan(h);
    h->create_offsets = nullptr;
    // per-segment stream bits for the cost model's features
    for (auto &s : h->segs)
      if (s.region == 0) s.bits = g->offsets[s.end] - g->offsets[s.begin];
    check(h, cudaStreamSynchronize(h->stream), "create");
    lpa_status st = lpa_init_labels(h);
    if (st != LPA_OK) throw Fail{st, h->last_error};
  } catch (const Fail &f) {
    lpa_status st = f.st;
    std::fprintf(stderr, "lpa_create: %s\n", f.msg.c_str());
    lpa_destroy(h);
    return st;
  }
  *out = h;
  return LPA_OK;
}

lpa_status lpa_destroy(lpa_handle *h) {
  if (!h) return LPA_ERR_INVALID_ARG;
  if (h->stream) cudaStreamSynchronize(h->stream);
  lpa_rt_destroy_graph(h);
  h->plan_builder.release();
  for (void *p : h->allocations) cudaFree(p);
  h->allocations.clear();
  if (h->h_pinned) cudaFreeHost(h->h_pinned);
  if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);
  if (h->h_wpinned) cudaFreeHost(h->h_wpinned);
  for (int b = 0; b < 2; b++) {
    if (h->ev_ready[b]) cudaEventDestroy(h->ev_ready[b]);
    if (h->ev_free[b]) cudaEventDestroy(h->ev_free[b]);
  }
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  for (auto &e : h->ev)
    if (e) cudaEventDestroy(e);
  lpa_learner_free(h);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  cudaGetLastError();
  delete h;
  return LPA_OK;
}

lpa_status lpa_get_info(lpa_handle *h, lpa_info *info) {
  if (!h || !info) return LPA_ERR_INVALID_ARG;
  std::memset(info, 0, sizeof(*info));
  info->num_vertices = h->n;
  info->num_compressed = h->n_c;
  info->num_arcs = h->m;
  info->num_small_arcs = h->m_small;
  info->stream_bits = h->total_bits;
  info->num_segments = h->segs.size();
  info->max_degree = h->max_deg;
  const uint64_t n_s = h->n - h->n_c;
  // bitstream + 8(n_c+1) offsets + 4 n_c ids + 4(n_s+1) + 4 m_s small CSR
  // + 4 n degrees + 4 n label reads + 4 n label writes
  info->bytes_algorithmic = (h->total_bits + 7) / 8 + 8 * (h->n_c + 1) + 4 * h->n_c + 4 * (n_s + 1) +
                            4 * h->m_small + 12 * h->n;
  info->device_bytes = h->device_bytes;
  return LPA_OK;
}

const char *lpa_last_error(lpa_handle *h) { return h ? h->last_error.c_str() : "null handle"; }

lpa_status lpa_init_labels(lpa_handle *h) {
  if (!h) return LPA_ERR_INVALID_ARG;
  try {
    check(h, cudaSetDevice(h->device), "cudaSetDevice");
    const int blocks = int(std::min<uint64_t>((h->n + 255) / 256, uint64_t(h->num_sms) * 8));
    k_init_labels<<<std::max(1, blocks), 256, 0, h->stream>>>(h->d_lab[0], h->d_lab[1], h->n);
    check(h, cudaGetLastError(), "init labels");
    h->cur = 0;
    h->iterations = 0;
    h->history.clear();
    check(h, cudaStreamSynchronize(h->stream), "init labels");
  } catch (const Fail &f) {
    return guard(h, f);
  }
  return LPA_OK;
}

lpa_status lpa_set_labels(lpa_handle *h, const uint32_t *host, size_t n) {
  if (!h || !host || n != h->n) return LPA_ERR_INVALID_ARG;
  try {
    check(h, cudaSetDevice(h->device), "cudaSetDevice");
    // both buffers: vertices without neighbours are never rewritten
    check(h, cudaMemcpyAsync(h->d_lab[0], host, n * 4, cudaMemcpyHostToDevice, h->stream), "set labels");
    check(h, cudaMemcpyAsync(h->d_lab[1], h->d_lab[0], n * 4, cudaMemcpyDeviceToDevice, h->stream), "set labels");
    check(h, cudaStreamSynchronize(h->stream), "set labels");
    h->cur = 0;
    h->iterations = 0;
    h->history.clear();
  } catch (const Fail &f) {
    return guard(h, f);
  }
  return LPA_OK;
}


lpa_status lpa_iterate(lpa_handle *h, uint64_t *changed_out) {
  if (!h) return LPA_ERR_INVALID_ARG;
  try {
    check(h, cudaSetDevice(h->device), "cudaSetDevice");
    lpa_learner_before_iteration(h);
    unsigned long long *slot = h->d_changed;
    check(h, cudaMemsetAsync(slot, 0, sizeof(unsigned long long), h->stream), "clear counter");
    const size_t slots = h->streamed ? std::max<size_t>(1, h->ranges.size()) : 1;  // a counter block per range
    check(h, cudaMemsetAsync(h->d_work, 0, kWorkCounters * slots * sizeof(uint32_t), h->stream), "clear work counters");
    enqueue_iteration(h, slot, h->d_work);
    check(h, cudaGetLastError(), "iteration launch");
    check(h, cudaMemcpyAsync(h->h_pinned, slot, sizeof(unsigned long long), cudaMemcpyDeviceToHost, h->stream),
          "read counter");
    lpa_status st = take_device_error(h);  // synchronises
    if (st != LPA_OK) return st;
    h->last_changed = h->h_pinned[0];
    h->history.push_back(h->last_changed);
    h->iterations++;
    collect_times(h);
    lpa_learner_after_iteration(h);
    if (h->opts.verbose)
      std::printf("%llu: %f (ms), updated %llu\n", (unsigned long long)h->iterations, h->last_iter_ms,
                  (unsigned long long)h->last_changed);
    if (changed_out) *changed_out = h->last_changed;
  } catch (const Fail &f) {
    return guard(h, f);
  }
  return LPA_OK;
}


lpa_status lpa_run(lpa_handle *h, int max_iter, int early_exit, int *iters_done) {
  if (!h || max_iter < 0) return LPA_ERR_INVALID_ARG;
  if (iters_done) *iters_done = 0;
  int done = 0;
  while (done < max_iter && !lpa_learner_settled(h)) {  // the cost model learns on host-driven iterations
    uint64_t ch = 0;
    lpa_status st = lpa_iterate(h, &ch);
    if (st != LPA_OK) return st;
    done++;
    if (early_exit && ch == 0) {
      if (iters_done) *iters_done = done;
      return LPA_OK;
    }
  }
  if (h->streamed) {  // the copies of the ranges run from the host loop
    while (done < max_iter) {
      uint64_t ch = 0;
      lpa_status st = lpa_iterate(h, &ch);
      if (st != LPA_OK) return st;
      done++;
      if (early_exit && ch == 0) break;
    }
    if (iters_done) *iters_done = done;
    return LPA_OK;
  }
  int rest = 0;
  lpa_status st = lpa_run_graph(h, max_iter - done, early_exit != 0, &rest);
  if (iters_done) *iters_done = done + rest;
  return st;
}

lpa_status lpa_get_changed_history(lpa_handle *h, uint64_t *out, size_t count) {
  if (!h || (!out && count)) return LPA_ERR_INVALID_ARG;
  if (count > h->history.size()) return LPA_ERR_INVALID_ARG;
  const size_t base = h->history.size() - count;
  for (size_t i = 0; i < count; i++) out[i] = h->history[base + i];
  return LPA_OK;
}

lpa_status lpa_get_labels(lpa_handle *h, uint32_t *host_out, size_t n) {
  if (!h || !host_out || n != h->n) return LPA_ERR_INVALID_ARG;
  try {
    check(h, cudaSetDevice(h->device), "cudaSetDevice");
    check(h, cudaMemcpyAsync(host_out, h->d_lab[h->cur], n * 4, cudaMemcpyDeviceToHost, h->stream), "get labels");
    check(h, cudaStreamSynchronize(h->stream), "get labels");
  } catch (const Fail &f) {
    return guard(h, f);
  }
  return LPA_OK;
}

lpa_status lpa_get_stats(lpa_handle *h, lpa_stats *st) {
  if (!h || !st) return LPA_ERR_INVALID_ARG;
  std::memset(st, 0, sizeof(*st));
  st->iterations = h->iterations;
  st->last_changed = h->last_changed;
  st->last_iter_ms = h->last_iter_ms;
  st->launches = h->launches;
  st->decode_ms = h->decode_ms;
  st->stream_ranges = h->streamed ? h->ranges.size() : 0;
  st->stream_bytes = h->streamed_bytes;
  st->iterate_ms = h->iterate_ms;
  st->count_ms = h->count_ms;
  st->packed_ms = h->packed_ms;
  for (int v = 0; v < 4; v++) st->variant_ms[v] = h->variant_ms[v];
  for (size_t s = 0; s < h->segs.size(); s++) {
    st->variant_segments[h->variant[s]]++;
    st->variant_arcs[h->variant[s]] += h->segs[s].arcs;
  }
  lpa_learner_stats(h, st);
  return LPA_OK;
}

lpa_status lpa_get_degrees(lpa_handle *h, uint32_t *deg_out, size_t n) {
  if (!h || !deg_out || n != h->n) return LPA_ERR_INVALID_ARG;
  std::memcpy(deg_out, h->h_deg.data(), n * sizeof(uint32_t));
  return LPA_OK;
}

lpa_status lpa_decode_csr(lpa_handle *h, uint64_t *row_out, uint32_t *clm_out) {
  if (!h || !row_out || (!clm_out && h->m)) return LPA_ERR_INVALID_ARG;
  try {
    check(h, cudaSetDevice(h->device), "cudaSetDevice");
    ensure_two_pass_scratch(h);
    std::vector<uint64_t> off(h->n + 1, 0);
    for (uint64_t p = 0; p < h->n; p++) off[p + 1] = off[p] + h->h_deg[p];
    std::vector<uint32_t> ids(off[h->n_c]);
    DecodeArgs a{};
    a.g = dev_graph(h);
    a.pos_list = nullptr;
    a.arc_off = h->d_arc_off;
    a.err = h->d_err;
    auto decode = [&](uint64_t p0, uint64_t p1) {
      a.pos_begin = p0;
      a.n_pos = p1 - p0;
      const int blocks = int(std::max<uint64_t>(1, std::min<uint64_t>((a.n_pos + 255) / 256, uint64_t(h->num_sms) * 8)));
      if (a.n_pos) k_decode_positions<<<blocks, 256, 0, h->stream>>>(a);
      check(h, cudaGetLastError(), "decode launch");
      return take_device_error(h);
    };
    if (h->streamed) {  // range by range through one stream buffer and the scratch
      for (const StreamRange &r : h->ranges) {
        if (r.p1 <= r.p0) continue;
        a.g.words = stage_words(h, 0, r.w0, r.w1, h->stream);
        a.out = scratch_base(h, r.a0);
        lpa_status st = decode(r.p0, r.p1);
        if (st != LPA_OK) return st;
        if (r.a1 > r.a0)
          check(h, cudaMemcpy(ids.data() + r.a0, h->d_scratch + (r.a0 & 3u), (r.a1 - r.a0) * 4, cudaMemcpyDeviceToHost),
                "read decode");
      }
    } else {
      a.out = h->d_scratch;
      lpa_status st = decode(0, h->n_c);
      if (st != LPA_OK) return st;
      check(h, cudaMemcpy(ids.data(), h->d_scratch, ids.size() * 4, cudaMemcpyDeviceToHost), "read decode");
    }
    std::vector<uint32_t> verts(h->n);
    check(h, cudaMemcpy(verts.data(), h->d_vertices, h->n * 4, cudaMemcpyDeviceToHost), "read vertices");
    std::vector<uint32_t> sm_off(h->n - h->n_c + 1, 0), sm_nbr(h->m_small);
    if (h->n > h->n_c)
      check(h, cudaMemcpy(sm_off.data(), h->d_small_off, sm_off.size() * 4, cudaMemcpyDeviceToHost), "read small");
    if (h->m_small)
      check(h, cudaMemcpy(sm_nbr.data(), h->d_small_nbr, sm_nbr.size() * 4, cudaMemcpyDeviceToHost), "read small");
    std::vector<uint64_t> deg_by_id(h->n + 1, 0);
    for (uint64_t p = 0; p < h->n; p++) deg_by_id[verts[p]] = h->h_deg[p];
    row_out[0] = 0;
    for (uint64_t v = 0; v < h->n; v++) row_out[v + 1] = row_out[v] + deg_by_id[v];
    for (uint64_t p = 0; p < h->n; p++) {
      const uint32_t v = verts[p];
      const uint32_t *src = p < h->n_c ? ids.data() + off[p] : sm_nbr.data() + sm_off[p - h->n_c];
      std::memcpy(clm_out + row_out[v], src, size_t(h->h_deg[p]) * 4);
    }
  } catch (const Fail &f) {
    return guard(h, f);
  }
  return LPA_OK;
}

lpa_status lpa_set_dispatch(lpa_handle *h, int dispatch, int force_variant) {
  if (!h || dispatch < 0 || dispatch > 2 || force_variant < 0 || force_variant > 3) return LPA_ERR_INVALID_ARG;
  try {
    check(h, cudaSetDevice(h->device), "cudaSetDevice");
    h->opts.dispatch = dispatch;
    h->opts.force_variant = force_variant;
    if (dispatch == LPA_DISPATCH_LEARNED && h->opts.record_timings < 1) h->opts.record_timings = 1;
    lpa_learner_reset(h);
    apply_dispatch(h, dispatch == LPA_DISPATCH_FORCE ? LPA_DISPATCH_FORCE : LPA_DISPATCH_FIXED, force_variant);
    check(h, cudaStreamSynchronize(h->stream), "dispatch");
  } catch (const Fail &f) {
    return guard(h, f);
  }
  return LPA_OK;
}

static bool tune_valid(const lpa_tune &t) {
  return t.group_positions >= 1 && t.group_positions <= 32 && t.warp_positions >= 1 && t.warp_positions <= 32 &&
         t.warp_max_degree >= 32 && t.warp_max_degree <= kCountWarpMax && t.warp_claim >= 1 && t.warp_claim <= 8 &&
         t.bulk_stage <= 1 && t.gather_cache <= 2 && t.stage_stream <= 2;
}

// One iteration from the current labels, repeated; the labels are left as
// they were (an iteration reads one buffer and writes the other, and the
// buffer pointer is put back).  Returns the least kernel busy time (ms) on
// the GPU clock, or a negative value when an iteration failed.
static double tune_trial(lpa_handle *h, int repeats) {
  const int cur = h->cur;
  double best = -1;
  h->measure_busy = true;
  for (int r = 0; r < repeats; r++) {
    check(h, cudaMemsetAsync(h->d_ktime, 0xFF, kBusyKernels * sizeof(unsigned long long), h->stream), "clear spans");
    check(h, cudaMemsetAsync(h->d_ktime + kBusyKernels, 0, kBusyKernels * sizeof(unsigned long long), h->stream),
          "clear spans");
    check(h, cudaMemsetAsync(h->d_changed, 0, sizeof(unsigned long long), h->stream), "clear counter");
    const size_t slots = h->streamed ? std::max<size_t>(1, h->ranges.size()) : 1;
    check(h, cudaMemsetAsync(h->d_work, 0, kWorkCounters * slots * sizeof(uint32_t), h->stream), "clear work counters");
    enqueue_iteration(h, h->d_changed, h->d_work);
    h->cur = cur;
    check(h, cudaGetLastError(), "tuning iteration");
    if (take_device_error(h) != LPA_OK) {
      h->measure_busy = false;
      return -1;
    }
    unsigned long long span[2 * kBusyKernels];
    check(h, cudaMemcpy(span, h->d_ktime, sizeof(span), cudaMemcpyDeviceToHost), "read spans");
    double busy = 0;
    for (int k = 0; k < kBusyKernels; k++)
      if (span[kBusyKernels + k] > span[k]) busy += double(span[kBusyKernels + k] - span[k]) * 1e-6;
    if (best < 0 || busy < best) best = busy;
  }
  h->measure_busy = false;
  return best;
}

// The cache key: GPU, graph, sketch threshold and plan.
static std::string tune_key(const lpa_handle *h) {
  cudaDeviceProp pr{};
  if (cudaGetDeviceProperties(&pr, h->device) != cudaSuccess) cudaGetLastError();
  std::string gpu = pr.name;
  for (char &ch : gpu)
    if (ch == ' ' || ch == '|') ch = '_';
  uint64_t fnv = 1469598103934665603ull;
  for (uint8_t v : h->variant) fnv = (fnv ^ v) * 1099511628211ull;
  uint64_t arcs = 0;
  for (const auto &sg : h->segs) arcs += sg.arcs;
  char buf[512];
  std::snprintf(buf, sizeof(buf), "v5|%s|sm%d|n%llu|nc%llu|arcs%llu|cms%u|plan%016llx", gpu.c_str(), pr.multiProcessorCount,
                (unsigned long long)h->n, (unsigned long long)h->n_c, (unsigned long long)arcs,
                h->opts.cms_threshold, (unsigned long long)fnv);
  return buf;
}

lpa_status lpa_get_tune(lpa_handle *h, lpa_tune *out) {
  if (!h || !out) return LPA_ERR_INVALID_ARG;
  *out = h->tune;
  return LPA_OK;
}

lpa_status lpa_set_tune(lpa_handle *h, const lpa_tune *t) {
  if (!h || !t || !tune_valid(*t)) return LPA_ERR_INVALID_ARG;
  try {
    check(h, cudaSetDevice(h->device), "cudaSetDevice");
    h->tune = *t;
    lpa_rt_apply_variants(h);
  } catch (const Fail &f) {
    return guard(h, f);
  }
  return LPA_OK;
}

lpa_status lpa_autotune(lpa_handle *h, const char *cache_path, int repeats, lpa_tune *out) {
  if (!h) return LPA_ERR_INVALID_ARG;
  if (repeats <= 0) repeats = 2;
  try {
    check(h, cudaSetDevice(h->device), "cudaSetDevice");
    const std::string key = tune_key(h);
    bool found = false;
    if (cache_path) {
      std::ifstream in(cache_path);
      std::string line;
      while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::string k;
        lpa_tune t{};
        if (ls >> k >> t.group_positions >> t.warp_positions >> t.warp_max_degree >> t.warp_claim >> t.bulk_stage >>
                t.gather_cache >> t.stage_stream &&
            k == key && tune_valid(t)) {
          h->tune = t;
          found = true;
        }
      }
    }
    if (found) {
      lpa_rt_apply_variants(h);
    } else if (h->n_cblock + h->n_cwarp > 0) {
      // coordinate descent, two sweeps; a candidate must win by 0.5 %
      lpa_tune best = h->tune;
      double best_ms = tune_trial(h, repeats);
      if (best_ms < 0) throw Fail{LPA_ERR_CUDA, "autotune: " + h->last_error};
      static const uint32_t groups[] = {8, 16, 24, 32}, warps[] = {1, 2, 4, 8, 16},
                            degs[] = {63, 127, 255, kCountWarpMax}, claims[] = {1, 2, 4, 8}, flags[] = {0, 1, 2};
      for (int sweep = 0; sweep < 2; sweep++) {
        for (int knob = 0; knob < 7; knob++) {
          const uint32_t *vals = knob == 0 ? groups : knob == 1 ? warps : knob == 2 ? degs : knob == 3 ? claims : flags;
          const int nv = knob == 1 ? 5 : knob == 4 ? 2 : knob >= 5 ? 3 : 4;
          for (int i = 0; i < nv; i++) {
            lpa_tune cand = best;
            uint32_t &slot = knob == 0 ? cand.group_positions
                             : knob == 1 ? cand.warp_positions
                             : knob == 2 ? cand.warp_max_degree
                             : knob == 3 ? cand.warp_claim
                             : knob == 4 ? cand.bulk_stage
                             : knob == 5 ? cand.gather_cache
                                         : cand.stage_stream;
            if (slot == vals[i]) continue;
            slot = vals[i];
            h->tune = cand;
            lpa_rt_apply_variants(h);
            const double ms = tune_trial(h, repeats);
            if (ms < 0) throw Fail{LPA_ERR_CUDA, "autotune: " + h->last_error};
            if (ms < best_ms * 0.995) {
              best = cand;
              best_ms = ms;
            }
          }
        }
      }
      h->tune = best;
      lpa_rt_apply_variants(h);
      if (cache_path) {
        std::ofstream o(cache_path, std::ios::app);
        o << key << ' ' << best.group_positions << ' ' << best.warp_positions << ' ' << best.warp_max_degree << ' '
          << best.warp_claim << ' ' << best.bulk_stage << ' ' << best.gather_cache << ' ' << best.stage_stream << ' '
          << best_ms << '\n';
      }
    }
    if (out) *out = h->tune;
  } catch (const Fail &f) {
    h->measure_busy = false;
    return guard(h, f);
  }
  return LPA_OK;
}

lpa_status lpa_set_plan(lpa_handle *h, const uint8_t *variant, size_t count) {
  if (!h || !variant || count != h->segs.size()) return LPA_ERR_INVALID_ARG;
  for (size_t s = 0; s < count; s++)
    if (variant[s] > 3 || !variant_capable(variant[s], h->segs[s], h->opts.cms_threshold)) return LPA_ERR_INVALID_ARG;
  try {
    check(h, cudaSetDevice(h->device), "cudaSetDevice");
    h->opts.dispatch = LPA_DISPATCH_FORCE;
    lpa_learner_reset(h);
    h->variant.assign(variant, variant + count);
    lpa_rt_apply_variants(h);
    check(h, cudaStreamSynchronize(h->stream), "plan");
  } catch (const Fail &f) {
    return guard(h, f);
  }
  return LPA_OK;
}

lpa_status lpa_get_capable(lpa_handle *h, uint8_t *mask, size_t count) {
  if (!h || !mask || count != h->segs.size()) return LPA_ERR_INVALID_ARG;
  for (size_t s = 0; s < count; s++) {
    uint8_t m = 0;
    for (int v = 0; v < kNumVariants; v++)
      if (variant_capable(v, h->segs[s], h->opts.cms_threshold)) m |= uint8_t(1u << v);
    mask[s] = m;
  }
  return LPA_OK;
}

lpa_status lpa_get_segments(lpa_handle *h, uint32_t *begin, uint32_t *end, uint8_t *bucket, uint8_t *variant,
                            size_t count) {
  if (!h || count != h->segs.size()) return LPA_ERR_INVALID_ARG;
  for (size_t s = 0; s < count; s++) {
    if (begin) begin[s] = h->segs[s].begin;
    if (end) end[s] = h->segs[s].end;
    if (bucket) bucket[s] = h->segs[s].bucket;
    if (variant) variant[s] = h->variant[s];
  }
  return LPA_OK;
}

}  // extern "C"

// Internal hooks used by the dispatch and graph-loop modules.
void lpa_rt_enqueue_iteration(lpa_handle *h, unsigned long long *changed, uint32_t *work) {
  enqueue_iteration(h, changed, work);
}
void lpa_rt_apply_variants(lpa_handle *h) {
  bool any_two = false;
  for (auto v : h->variant) any_two |= v == LPA_VARIANT_TWO_PASS;
  if (any_two) ensure_two_pass_scratch(h);
  upload_lists(h);
}
lpa_status lpa_rt_take_error(lpa_handle *h) { return take_device_error(h); }
