// Label-propagation kernels for sm_100a.
//
// One synchronous iteration reads lab_in and writes lab_out (double-buffered)
// for every vertex of degree > 0.  The update rule: the most frequent
// neighbour label, the smallest label on ties; vertices with degree >=
// cms_thr (cms_thr != 0) use a depth-4, width-1024 count-min sketch with
// seeded cm_hash rows (include/cms.cuh:96-132) and take the argmax of the
// sketch estimate over their neighbour labels, smallest label on ties.
//
// k_iterate is a persistent kernel fed by two device work queues:
//   * heavy items (block variant, and two-pass segments above the warp
//     limit), taken by a whole block, largest first: 256-bit segments decode in
//     parallel (one thread each), ids are staged in shared memory, labels are
//     gathered with many loads in flight, then counted in a shared (or global)
//     table or the sketch;
//   * light chunks of up to 32 consecutive positions, taken by one warp: each
//     lane decodes one vertex into the warp's staging area, the warp gathers
//     all labels at once, then counts per vertex (one vertex per round, or
//     several vertices per round for degrees <= 32).
// Every loop is bounded by the bits it consumes; malformed input sets the
// error word instead of trapping.
#include <type_traits>

#include "lp_kernels.cuh"
#include "noalloc.cuh"

namespace lpa_dev {

namespace {

// Epoch ranges of the shared tables: warp tables use [1, kLightEpochs), the
// block table [kLightEpochs, 65536), so a slot left by one mode never matches
// the other.
constexpr uint32_t kLightEpochs = 32768;
constexpr uint32_t kHeavyEpochFirst = 32768;

__device__ __forceinline__ uint32_t next_pow2(uint32_t x) { return x <= 1 ? 1u : (1u << (32 - __clz(x - 1))); }

struct Ctx {
  const uint32_t *lab_in;
  uint32_t *lab_out;
  unsigned long long *changed;
  uint32_t it;
  bool coherent;  // labels may change within the launch (batched graphs): read them through L2
};

// A label read: the non-coherent path when labels are fixed for the whole
// launch, else an L2 (ld.global.cg) read.
__device__ __forceinline__ uint32_t ld_label(const Ctx &c, uint32_t i) {
  return c.coherent ? __ldcg(c.lab_in + i) : __ldg(c.lab_in + i);
}

// An L2 cache policy that evicts the lines it is given last, and a load
// through L2 only (ld.global.cg) under such a policy.
__device__ __forceinline__ uint64_t l2_evict_last_policy() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint32_t ld_cg_keep(const uint32_t *q, uint64_t pol) {
  uint32_t v;
  asm("ld.global.cg.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(q), "l"(pol));
  return v;
}

// A neighbour's label in a random gather: the lowest kHotIds ids (the hubs,
// in BFS order) through L1, every other id through L2 only, so that the
// scattered reads do not push the hot labels out of L1.
__device__ __forceinline__ uint32_t ld_label_gather(const Ctx &c, uint32_t i) {
  return (!c.coherent && i < kHotIds) ? __ldg(c.lab_in + i) : __ldcg(c.lab_in + i);
}

__device__ __forceinline__ Ctx resolve(const IterArgs &a) {
  Ctx c;
  c.it = iter_index(a);
  const uint32_t par = (a.parity0 + c.it) & 1u;
  c.lab_in = par ? a.labs1 : a.labs0;
  c.lab_out = par ? a.labs0 : a.labs1;
  c.changed = a.changed + (a.it_dev ? c.it : 0u);
  c.coherent = false;
  return c;
}

__device__ __forceinline__ void flush_changed(unsigned long long *counter, unsigned long long mine) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(kFull, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(counter, mine);
}

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, uint32_t lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t t = __shfl_up_sync(kFull, v, o);
    if (lane >= uint32_t(o)) v += t;
  }
  return v;
}

struct BlockSh {
  uint32_t pref[kThreads + 1];
  uint32_t left[kThreads];
  uint32_t wsum[kWarps];
  uint64_t red[kWarps];
  uint64_t ibase, rbase, last_end;
  uint32_t nseg_i, nseg_r, item, items, bad;
  uint32_t spill_n;  // labels a hub has written to its spill area so far
  uint32_t hepoch;  // epoch of the block's exact table
};

// Block-wide exclusive scan of v into sh.pref; returns the total.
__device__ __forceinline__ uint32_t block_scan(BlockSh &sh, uint32_t v) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t incl = warp_incl_scan(v, lane);
  if (lane == 31) sh.wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    const uint32_t w = lane < kWarps ? sh.wsum[lane] : 0u;
    const uint32_t wi = warp_incl_scan(w, lane);
    if (lane < kWarps) sh.wsum[lane] = wi - w;
    if (lane == kWarps - 1) sh.pref[kThreads] = wi;
  }
  __syncthreads();
  sh.pref[threadIdx.x] = incl - v + sh.wsum[warp];
  __syncthreads();
  return sh.pref[kThreads];
}

// ------------------------------------------------------------ consumers ---
// A warp-uniform run of one label: a step whose real labels all equal the
// run's label only adds to the run's count (two ballots), so a vertex whose
// neighbours share one label touches its table once per label change, not
// once per step.  extend() is called by all 32 lanes.
struct WarpRun {
  uint32_t lab = kFull, cnt = 0;
  __device__ __forceinline__ bool extend(bool ok, uint32_t l) {
    const uint32_t okm = __ballot_sync(kFull, ok);
    if (__ballot_sync(kFull, ok && l == lab) != okm) return false;
    cnt += __popc(okm);
    return true;
  }
  // starts a new run at the label of the step's first real lane (the step
  // itself is counted by the caller)
  __device__ __forceinline__ void restart(bool ok, uint32_t l) {
    const uint32_t okm = __ballot_sync(kFull, ok);
    lab = __shfl_sync(kFull, l, __ffs(okm) - 1);
    cnt = 0;
  }
};

// Sinks are called warp-synchronously by every lane; ok marks a real label.
// The exact tables fold lanes holding the same label first (warp_merge), so a
// step whose lanes share a label touches the table once.
struct ExactSink {  // global table (key/count arrays, cleared after use)
  uint32_t *keys, *cnts, cap;
  __device__ __forceinline__ void operator()(bool ok, uint32_t lab) const {
    const uint32_t w = warp_merge(ok, lab);
    if (w) table_add(keys, cnts, cap, lab, w);
  }
};

struct EpochSink {  // shared epoch table with a running argmax per thread
  EpochTable et;
  uint64_t *best;
  __device__ __forceinline__ void operator()(bool ok, uint32_t lab) const {
    const uint32_t w = warp_merge(ok, lab);
    if (w) {
      const uint64_t cand = pack_best(et.insert(lab, w), lab);
      if (cand > *best) *best = cand;
    }
  }
};

// Every lane adds its own label: the shared-memory atomics absorb the
// conflicts of lanes holding the same label for less than folding them first
// costs (fixed plan at R-MAT scale 24: 13.48 -> 13.02 ms per iteration).
struct CmsAddSink {
  uint32_t *cms;
  const uint32_t *seeds;
  uint32_t base;  // label_base of the vertex
  __device__ __forceinline__ void operator()(bool ok, uint32_t lab) const {
    if (ok) {
#pragma unroll
      for (int r = 0; r < kCmsDepth; r++)
        atomicAdd(&cms[r * kCmsWidth + (cm_hash(r, (lab - base) ^ seeds[r]) & (kCmsWidth - 1))], 1u);
    }
  }
};

// Passes every label on to `inner` and also writes it to spill[0..cap), one
// reservation per 32 labels (warp-synchronous, like every sink): the sketch's
// second pass over a decoded hub then reads the labels back instead of
// decoding the hub again.
template <class Sink>
struct SpillSink {
  Sink inner;
  uint32_t *spill;
  uint32_t cap;
  uint32_t *count;  // shared
  __device__ __forceinline__ void operator()(bool ok, uint32_t lab) const {
    inner(ok, lab);
    const uint32_t m = __ballot_sync(kFull, ok);
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t base = 0;
    if (lane == 0 && m) base = atomicAdd(count, uint32_t(__popc(m)));
    base = __shfl_sync(kFull, base, 0);
    const uint32_t at = base + uint32_t(__popc(m & ((1u << lane) - 1u)));
    if (ok && at < cap) spill[at] = lab;
  }
};

// Second sketch pass: read-only, so every lane looks up its own label.
struct CmsBestSink {
  const uint32_t *cms;
  const uint32_t *seeds;
  uint32_t base;
  uint64_t *best;
  __device__ __forceinline__ void operator()(bool ok, uint32_t lab) const {
    if (ok) {
      // est <= the first row's counter: a label whose first counter cannot
      // beat this lane's best is not looked up further (fixed plan at R-MAT
      // scale 24: -0.1 ms per iteration)
      uint32_t est = cms[cm_hash(0, (lab - base) ^ seeds[0]) & (kCmsWidth - 1)];
      if (pack_best(est, lab) > *best) {
#pragma unroll
        for (int r = 1; r < kCmsDepth; r++) {
          const uint32_t v = cms[r * kCmsWidth + (cm_hash(r, (lab - base) ^ seeds[r]) & (kCmsWidth - 1))];
          est = v < est ? v : est;
        }
        const uint64_t cand = pack_best(est, lab);
        if (cand > *best) *best = cand;
      }
    }
  }
};

// Labels of the global ids src[0..total) into stage (src_labels: src holds
// the labels themselves).
__device__ __forceinline__ void block_gather_from(uint32_t *stage, const uint32_t *__restrict__ src, uint32_t total,
                                                  const Ctx &c, bool src_labels) {
  for (uint32_t k0 = threadIdx.x; k0 < total; k0 += 4 * kThreads) {
    uint32_t v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t k = k0 + u * kThreads;
      v[u] = k >= total ? 0u : (src_labels ? __ldcs(src + k) : ld_label_gather(c, __ldg(src + k)));
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t k = k0 + u * kThreads;
      if (k < total) stage[k] = v[u];
    }
  }
}

// Labels src[0..total) from global memory (a hub's spill area), 4 loads per
// thread in flight, into sink; block-synchronous.
template <class Sink>
__device__ __forceinline__ void block_consume_global(const uint32_t *src, uint32_t total, const Sink &sink) {
  for (uint32_t k0 = 0; k0 < total; k0 += 4 * kThreads) {
    uint32_t v[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t k = k0 + u * kThreads + threadIdx.x;
      v[u] = k < total ? __ldcg(src + k) : 0u;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t k = k0 + u * kThreads + threadIdx.x;
      sink(k < total, v[u]);
    }
  }
}

template <class Sink>
__device__ __forceinline__ void block_consume_stage(const uint32_t *stage, uint32_t total, const Sink &sink) {
  for (uint32_t k0 = 0; k0 < total; k0 += kThreads) {
    const uint32_t k = k0 + threadIdx.x;
    const bool ok = k < total;
    sink(ok, ok ? stage[k] : 0u);
  }
}

// Feeds every neighbour label of position p to sink, block-synchronously.
// Returns true when all labels ended up in stage[0..d) (one chunk, no
// intervals), so a second pass can read them from there.
template <class Sink>
__device__ bool heavy_produce(const IterArgs &a, const Ctx &c, BlockSh &sh, uint32_t *stage, uint32_t p,
                              uint32_t node, uint32_t d, bool from_scratch, const Sink &sink) {
  const DevGraph &g = a.g;
  const uint32_t t = threadIdx.x;
  if (p >= g.n_c || from_scratch) {
    // contiguous: the small CSR's ids, or the labels the two-pass pre-pass wrote
    const bool labels = p < g.n_c && a.scratch_labels;
    const uint32_t *src = labels ? a.scratch + a.arc_off[p] : g.small_nbr + g.small_off[p - g.n_c];
    for (uint32_t c0 = 0; c0 < d; c0 += kStage) {
      const uint32_t cnt = min(kStage, d - c0);
      block_gather_from(stage, src + c0, cnt, c, labels);
      __syncthreads();
      block_consume_stage(stage, cnt, sink);
      __syncthreads();
    }
    return false;
  }
  const uint64_t end = g.offsets[p + 1];
  bool bad = false;
  uint32_t my_items = 0;
  if (t == 0) {
    BitReader r;
    r.seek(g.words, g.offsets[p]);
    uint32_t ns = r.segcnt(bad);
    if (bad || r.pos() > end || ns > (end - r.pos()) / kSegBits + 1) {
      bad = true;
      ns = 0;
    }
    sh.nseg_i = ns;
    sh.ibase = r.pos();
    sh.last_end = r.pos();
    sh.bad = bad ? 1u : 0u;
    sh.items = 0;
  }
  __syncthreads();
  const uint32_t nseg_i = sh.nseg_i;
  const uint64_t ibase = sh.ibase;
  // ---- interval section: pairs decoded one per thread per step, flattened block-wide
  for (uint32_t j0 = 0; j0 < nseg_i; j0 += kThreads) {
    const uint32_t j = j0 + t;
    bool has = j < nseg_i;
    BitReader r;
    uint32_t cnt = 0, cc = 0, left = 0;
    const uint64_t q = ibase + uint64_t(kSegBits) * j;
    if (has) {
      if (q >= end) {
        bad = true;
        has = false;
      } else {
        r.seek(g.words, q);
        cnt = r.gamma(bad);
      }
    }
    while (__syncthreads_or(has && cc < cnt)) {
      uint32_t len = 0;
      if (has && cc < cnt) {
        const uint32_t l = r.gamma(bad);
        left = (cc == 0) ? zigzag_first(node, l) : left + l + 1u;
        len = r.gamma(bad) + kMinItv;
        cc++;
        if (bad || r.pos() > end || uint64_t(left) + len > g.n) {
          bad = true;
          len = 0;
          cnt = cc;
        }
      }
      sh.left[t] = left;
      const uint32_t total = block_scan(sh, len);
      if (len) left += len;
      for (uint32_t i0 = 0; i0 < total; i0 += 4 * kThreads) {
        uint32_t lab[4];
        bool ok[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const uint32_t i = i0 + u * kThreads + t;
          ok[u] = i < total;
          lab[u] = 0;
          if (ok[u]) {
            uint32_t lo = 0, hi = kThreads - 1;
            while (lo < hi) {
              const uint32_t mid = (lo + hi + 1) >> 1;
              if (sh.pref[mid] <= i) lo = mid;
              else hi = mid - 1;
            }
            lab[u] = ld_label(c, sh.left[lo] + (i - sh.pref[lo]));
            my_items++;
          }
        }
#pragma unroll
        for (int u = 0; u < 4; u++) sink(ok[u], lab[u]);
      }
      __syncthreads();
    }
    if (has && j == nseg_i - 1) sh.last_end = r.pos();
  }
  __syncthreads();
  // ---- residual section: every warp walks its own 256-bit segments (lane per
  // segment, 32 per round) through its slice of the staging area; warps only
  // meet again at the end.
  if (t == 0) {
    BitReader r;
    r.seek(g.words, sh.last_end);
    uint32_t ns = r.segcnt(bad);
    if (bad || r.pos() > end || ns > (end - r.pos()) / kSegBits + 1) {
      bad = true;
      ns = 0;
    }
    sh.nseg_r = ns;
    sh.rbase = r.pos();
    sh.last_end = r.pos();
  }
  __syncthreads();
  const uint32_t nseg_r = sh.nseg_r;
  const uint64_t rbase = sh.rbase;
  const uint32_t lane = t & 31u, warp = t >> 5;
  uint32_t *wst = stage + warp * kWarpStage;
  bool single = true;  // this warp's labels all sit in its slice after one batch
  uint32_t staged = 0;
  int batches = 0;
  for (uint32_t j0 = warp * 32u; j0 < nseg_r; j0 += kWarps * 32u) {
    const uint32_t j = j0 + lane;
    bool has = j < nseg_r;
    BitReader r;
    uint32_t cnt = 0;
    if (has) {
      const uint64_t q = rbase + uint64_t(kSegBits) * j;
      if (q >= end) {
        bad = true;
        has = false;
      } else {
        r.seek(g.words, q);
        cnt = r.gamma(bad);
        if (bad || cnt > kWarpStage) {
          bad = true;
          cnt = 0;
        }
      }
    }
    uint32_t done = ~__ballot_sync(kFull, has);
    while (done != kFull) {
      const bool pending = !((done >> lane) & 1u);
      const uint32_t sc = pending ? cnt : 0u;
      const uint32_t incl = warp_incl_scan(sc, lane);
      const bool in_batch = pending && incl <= kWarpStage;
      const uint32_t batch = __ballot_sync(kFull, in_batch);
      const uint32_t total = __shfl_sync(kFull, incl, 31 - __clz(batch));
      if (in_batch) {
        // ids are clamped to n - 1, so every gather stays in range; a
        // segment's ids ascend, so its last one is its largest, and it and the
        // segment's end are tested once, after the last code (the stream was
        // validated code by code when the handle was created)
        const uint32_t nmax = uint32_t(g.n - 1);
        uint32_t o = incl - sc, v = 0;
        if (cnt) {
          v = zigzag_first(node, r.zeta3(bad));
          wst[o++] = min(v, nmax);
        }
        for (uint32_t cc = 1; cc < cnt; cc++) {
          v += r.zeta3(bad) + 1u;
          wst[o++] = min(v, nmax);
        }
        if (cnt && (v > nmax || r.pos() > end)) bad = true;
        my_items += cnt;
        if (j == nseg_r - 1) sh.last_end = r.pos();
      }
      __syncwarp();
      for (uint32_t k0 = lane; k0 < total; k0 += 256) {
        uint32_t lv[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const uint32_t k = k0 + 32 * u;
          lv[u] = k < total ? ld_label_gather(c, wst[k]) : 0u;
        }
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const uint32_t k = k0 + 32 * u;
          if (k < total) wst[k] = lv[u];
        }
      }
      __syncwarp();
      for (uint32_t k0 = 0; k0 < total; k0 += 32) {
        const uint32_t k = k0 + lane;
        const bool ok = k < total;
        sink(ok, ok ? wst[k] : 0u);
      }
      __syncwarp();
      staged = total;
      batches++;
      done |= batch;
    }
  }
  if (batches > 1) single = false;
  if (my_items) atomicAdd(&sh.items, my_items);
  if (bad) sh.bad = 1;
  const bool all_single = __syncthreads_and(single) != 0;
  if (t == 0 && (sh.bad || sh.last_end != end || sh.items != d)) set_error(a.err, kErrBadStream);
  if (lane == 0) sh.wsum[warp] = staged;
  __syncthreads();
  return nseg_i == 0 && all_single;
}

// Second pass over labels left in the warps' slices by heavy_produce.
template <class Sink>
__device__ __forceinline__ void heavy_consume_staged(BlockSh &sh, const uint32_t *stage, const Sink &sink) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t *wst = stage + warp * kWarpStage;
  const uint32_t total = sh.wsum[warp];
  for (uint32_t k0 = 0; k0 < total; k0 += 32) {
    const uint32_t k = k0 + lane;
    const bool ok = k < total;
    sink(ok, ok ? wst[k] : 0u);
  }
}

// One heavy vertex by the whole block.
__device__ void heavy_vertex(const IterArgs &a, const Ctx &c, BlockSh &sh, uint32_t *stage, uint32_t *tab,
                             uint32_t seg, uint32_t p, bool from_scratch, unsigned long long &changed) {
  const DevGraph &g = a.g;
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint32_t node = g.vertices[p];
  const uint32_t d = g.deg[p];
  const uint32_t old = ld_label(c, node);
  if (a.cursor && from_scratch && p < g.n_c && t == 0) a.cursor[p] = 0u;  // the pre-pass's output cursor, for the next iteration
  if (d == 0) return;
  uint64_t best = 0;
  if (a.cms_thr != 0 && d >= a.cms_thr) {
    // the sketch shares its memory with the exact tables, whose slots are
    // never cleared: zero the counters first
    uint32_t *cms = tab;
    for (uint32_t i = t; i < kCmsDepth * kCmsWidth; i += kThreads) cms[i] = 0u;
    __syncthreads();
    const uint32_t lb = label_base(a, node);
    // a hub decoded here keeps its labels in the block's spill area (when it
    // fits), so the second pass reads them back instead of decoding again
    const bool decoded = p < g.n_c && !from_scratch;
    uint32_t *spill = (a.hub_spill && decoded && d <= a.hub_spill_words)
                          ? a.hub_spill + uint64_t(blockIdx.x) * a.hub_spill_words
                          : nullptr;
    if (t == 0) sh.spill_n = 0;
    __syncthreads();
    const CmsAddSink s1{cms, a.seeds, lb};
    const bool staged = spill ? heavy_produce(a, c, sh, stage, p, node, d, from_scratch,
                                              SpillSink<CmsAddSink>{s1, spill, d, &sh.spill_n})
                              : heavy_produce(a, c, sh, stage, p, node, d, from_scratch, s1);
    __syncthreads();
    CmsBestSink s2{cms, a.seeds, lb, &best};
    if (staged) heavy_consume_staged(sh, stage, s2);
    else if ((p >= g.n_c || from_scratch) && d <= kStage) block_consume_stage(stage, d, s2);
    else if (spill && sh.spill_n == d) block_consume_global(spill, d, s2);
    else heavy_produce(a, c, sh, stage, p, node, d, from_scratch, s2);
    __syncthreads();
    // leave no counter behind that an epoch table could read as its own slot
    for (uint32_t i = t; i < kCmsDepth * kCmsWidth; i += kThreads) cms[i] = 0u;
  } else if (d <= kBlockMaxSmemDeg) {
    unsigned long long *slots = reinterpret_cast<unsigned long long *>(tab);
    if (t == 0) {
      if (++sh.hepoch >= 65536u) sh.hepoch = 0;
    }
    __syncthreads();
    if (sh.hepoch == 0) {  // epochs used up: start the block table over
      for (uint32_t i = t; i < kTableSlots; i += kThreads) slots[i] = 0ull;
      __syncthreads();
      if (t == 0) sh.hepoch = kHeavyEpochFirst;
      __syncthreads();
    }
    const EpochTable et{slots, next_pow2(2 * d), sh.hepoch};
    heavy_produce(a, c, sh, stage, p, node, d, from_scratch, EpochSink{et, &best});
    __syncthreads();
  } else {
    const uint32_t cap = next_pow2(2 * d);
    if (a.gtab_slots == 0 || cap > a.gtab_slots) {
      if (t == 0) set_error(a.err, kErrCapacity);
      return;
    }
    uint32_t *keys = a.gtab + uint64_t(blockIdx.x) * 2 * a.gtab_slots;
    uint32_t *cnts = keys + a.gtab_slots;
    heavy_produce(a, c, sh, stage, p, node, d, from_scratch, ExactSink{keys, cnts, cap});
    __syncthreads();
    for (uint32_t i = t; i < cap; i += kThreads) {
      const uint32_t kk = keys[i];
      if (kk) {
        const uint64_t cand = pack_best(cnts[i], kk - 1u);
        best = cand > best ? cand : best;
        keys[i] = 0u;
        cnts[i] = 0u;
      }
    }
  }
  best = warp_max_u64(best);
  if (lane == 0) sh.red[warp] = best;
  __syncthreads();
  if (t == 0) {
    uint64_t b = 0;
    for (int w = 0; w < kWarps; w++) b = sh.red[w] > b ? sh.red[w] : b;
    const uint32_t nl = b ? best_label(b) : old;
    c.lab_out[node] = nl;
    changed += (nl != old);
    if (a.seg_changed && nl != old) atomicAdd(a.seg_changed + seg, 1u);
  }
  __syncthreads();
}

// Decodes the compressed vertices of a warp batch into stage (ids).  Lane l
// owns the batch vertex in lane l: it reads that vertex's section headers and
// writes its interval items (lane per vertex); then the batch's residual
// segments are spread over the lanes (lane per 256-bit segment, 32 per
// round) and placed with warp prefix sums over the segments' item counts.
// Returns false (after filling every region with in-range ids) on a
// malformed stream.
__device__ bool warp_decode_batch(const DevGraph &g, uint32_t *stage, bool active, uint32_t p, uint32_t node,
                                  uint32_t d, uint32_t base, uint32_t lane) {  // stage: shared or global
  bool bad = false;
  uint32_t nres = 0, itv = 0;
  uint64_t rbase = 0, end = 0;
  if (active && d) {
    end = g.offsets[p + 1];
    BitReader r;
    r.seek(g.words, g.offsets[p]);
    uint32_t ns = r.segcnt(bad);
    const uint64_t ib = r.pos();
    uint64_t last = r.pos();
    if (bad || r.pos() > end || ns > (end - r.pos()) / kSegBits + 1) {
      bad = true;
      ns = 0;
    }
    for (uint32_t j = 0; j < ns && !bad; j++) {
      const uint64_t q = ib + uint64_t(kSegBits) * j;
      if (q >= end) {
        bad = true;
        break;
      }
      if (j) r.seek(g.words, q);
      const uint32_t cnt = r.gamma(bad);
      uint32_t left = 0;
      for (uint32_t c = 0; c < cnt && !bad; c++) {
        const uint32_t l = r.gamma(bad);
        left = (c == 0) ? zigzag_first(node, l) : left + l + 1u;
        const uint32_t len = r.gamma(bad) + kMinItv;
        if (bad || r.pos() > end || uint64_t(left) + len > g.n || uint64_t(itv) + len > d) {
          bad = true;
          break;
        }
        for (uint32_t k = 0; k < len; k++) stage[base + itv + k] = left + k;
        itv += len;
        left += len;
      }
      last = r.pos();
    }
    if (ns) r.seek(g.words, last);
    if (!bad) {
      nres = r.segcnt(bad);
      rbase = r.pos();
      if (bad || r.pos() > end || nres > (end - r.pos()) / kSegBits + 1) {
        bad = true;
        nres = 0;
      } else if (nres == 0 && r.pos() != end) {
        bad = true;
      }
    }
  }
  const uint32_t seg_incl = warp_incl_scan(nres, lane);
  const uint32_t seg_excl = seg_incl - nres;
  const uint32_t S = __shfl_sync(kFull, seg_incl, 31);
  uint32_t res_done = 0;
  for (uint32_t r0 = 0; r0 < S; r0 += 32) {
    const uint32_t f = r0 + lane;
    const bool has = f < S;
    // owner: the last lane whose first segment is <= f
    uint32_t lo = 0, hi = 31;
#pragma unroll
    for (int step = 0; step < 5; step++) {
      const uint32_t mid = (lo + hi + 1) >> 1;
      const uint32_t e = __shfl_sync(kFull, seg_excl, mid);
      if (e <= f) lo = mid;
      else hi = mid - 1;
    }
    const uint32_t o = lo;
    const uint32_t eo = __shfl_sync(kFull, seg_excl, o);
    const uint32_t no = __shfl_sync(kFull, nres, o);
    const uint64_t rb = __shfl_sync(kFull, rbase, o);
    const uint64_t en = __shfl_sync(kFull, end, o);
    const uint32_t ndo = __shfl_sync(kFull, node, o);
    const uint32_t bo = __shfl_sync(kFull, base, o);
    const uint32_t io = __shfl_sync(kFull, itv, o);
    const uint32_t dd = __shfl_sync(kFull, d, o);
    const uint32_t rdo = __shfl_sync(kFull, res_done, o);
    const uint32_t j = f - eo;
    BitReader rr;
    uint32_t cnt = 0;
    if (has) {
      const uint64_t q = rb + uint64_t(kSegBits) * j;
      if (q >= en) {
        bad = true;
      } else {
        rr.seek(g.words, q);
        cnt = rr.gamma(bad);
        if (bad || cnt > dd) {
          bad = true;
          cnt = 0;
        }
      }
    }
    const uint32_t c_incl = warp_incl_scan(cnt, lane);
    const uint32_t c_excl = c_incl - cnt;
    const uint32_t fo = (eo > r0 ? eo : r0) - r0;  // the owner's first lane in this round
    const uint32_t at_fo = __shfl_sync(kFull, c_excl, fo);
    if (has && !bad) {
      const uint32_t rel = io + rdo + (c_excl - at_fo);  // item offset inside the owner's region
      if (uint64_t(rel) + cnt > dd) {
        bad = true;
      } else {
        // clamped ids, one range and end test per segment (as heavy_produce)
        const uint32_t nmax = uint32_t(g.n - 1);
        uint32_t v = 0;
        if (cnt) {
          v = zigzag_first(ndo, rr.zeta3(bad));
          stage[bo + rel] = min(v, nmax);
        }
        for (uint32_t c = 1; c < cnt; c++) {
          v += rr.zeta3(bad) + 1u;
          stage[bo + rel + c] = min(v, nmax);
        }
        if (cnt && (v > nmax || rr.pos() > en)) bad = true;
      }
      if (j == no - 1 && rr.pos() != en) bad = true;
    }
    // owners advance by the items of their segments in this round
    const uint32_t fv = (seg_excl > r0 ? seg_excl : r0) - r0;
    const uint32_t lv_end = (seg_incl < r0 + 32 ? seg_incl : r0 + 32);
    const bool mine = nres && seg_incl > r0 && seg_excl < r0 + 32;
    const uint32_t lv = mine ? lv_end - r0 - 1 : 0u;
    const uint32_t a1 = __shfl_sync(kFull, c_incl, lv);
    const uint32_t a0 = __shfl_sync(kFull, c_excl, mine ? fv : 0u);
    if (mine) res_done += a1 - a0;
  }
  if (active && d && itv + res_done != d) bad = true;
  if (__any_sync(kFull, bad)) {
    if (active)
      for (uint32_t k = 0; k < d; k++) stage[base + k] = node;
    __syncwarp();
    return false;
  }
  return true;
}

// Up to 32 consecutive positions [p0, p1) by one warp.
__device__ void light_chunk(const IterArgs &a, const Ctx &c, uint32_t *stage, unsigned long long *slots,
                            uint32_t &epoch, uint32_t seg, uint32_t p0, uint32_t p1, int variant,
                            unsigned long long &changed) {
  const DevGraph &g = a.g;
  const uint32_t lane = threadIdx.x & 31u;
  constexpr uint32_t cap_stage = kWarpStage;
  const uint32_t p = p0 + lane;
  const bool valid = p < p1;
  const uint32_t node = valid ? g.vertices[p] : 0u;
  uint32_t d = valid ? g.deg[p] : 0u;
  const uint32_t old = valid ? ld_label(c, node) : 0u;
  const bool cgr = p0 < g.n_c;  // chunks never straddle the compressed / small boundary
  const bool decode = cgr && variant != kVarTwoPass;
  if (a.cursor && cgr && !decode && valid) a.cursor[p] = 0u;  // the pre-pass's output cursor, for the next iteration
  if (d > cap_stage || (variant == kVarPacked && d > kV2MaxDeg) || d > kV1MaxDeg) {
    set_error(a.err, kErrCapacity);
    d = 0;
  }
  // contiguous id source of the chunk when it is not decoded here
  const uint32_t *src = nullptr;
  if (!decode) src = cgr ? a.scratch + a.arc_off[p0] : g.small_nbr + g.small_off[p0 - g.n_c];
  uint32_t src_skip = 0;  // ids consumed by earlier batches of this chunk
  uint32_t done = ~__ballot_sync(kFull, valid);
  uint32_t my_changed = 0;
  while (done != kFull) {
    const bool pending = !((done >> lane) & 1u);
    const uint32_t sd = pending ? d : 0u;
    const uint32_t incl = warp_incl_scan(sd, lane);
    const bool in_batch = pending && incl <= cap_stage;
    const uint32_t batch = __ballot_sync(kFull, in_batch);
    const uint32_t lo = __ffs(batch) - 1, hi = 32 - __clz(batch);
    const uint32_t total = __shfl_sync(kFull, incl, hi - 1);
    const uint32_t base = incl - sd;
    // 1. ids: the batch decoded by all lanes together
    if (decode && !warp_decode_batch(g, stage, in_batch, p, node, d, base, lane) && lane == 0)
      set_error(a.err, kErrBadStream);
    __syncwarp();
    // 2. labels: every load of the batch in flight together
    for (uint32_t k0 = lane; k0 < total; k0 += 256) {
      uint32_t v[8];
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const uint32_t k = k0 + 32 * u;
        v[u] = k >= total ? 0u
                          : (decode ? ld_label_gather(c, stage[k])
                                    : (cgr && a.scratch_labels ? __ldcs(src + src_skip + k)
                                                               : ld_label_gather(c, __ldg(src + src_skip + k))));
      }
#pragma unroll
      for (int u = 0; u < 8; u++) {
        const uint32_t k = k0 + 32 * u;
        if (k < total) stage[k] = v[u];
      }
    }
    __syncwarp();
    // 3. count
    const uint32_t dmax = __reduce_max_sync(kFull, in_batch ? d : 0u);
    if (dmax <= 32 && (variant == kVarPacked || dmax <= 1)) {
      // several vertices per round: G lanes per vertex
      const uint32_t G = next_pow2(dmax);
      const uint32_t per = 32 / G;
      const uint32_t gl = lane / G, k = lane % G;
      const uint32_t gm = (G == 32) ? kFull : (((1u << G) - 1u) << (gl * G));
      for (uint32_t v0 = lo; v0 < hi; v0 += per) {
        const uint32_t vi = v0 + gl;
        const bool vin = vi < hi;
        const uint32_t srcl = vin ? vi : lo;
        const uint32_t dv = __shfl_sync(kFull, d, srcl);
        const uint32_t bv = __shfl_sync(kFull, base, srcl);
        const uint32_t nodev = __shfl_sync(kFull, node, srcl);
        const uint32_t oldv = __shfl_sync(kFull, old, srcl);
        const bool ok = vin && k < dv;
        const uint32_t lab = ok ? stage[bv + k] : kFull;
        const uint32_t cnt = group_counts(ok, lab, gm, gl);
        const uint32_t maxc = __reduce_max_sync(gm, cnt);
        const uint32_t bestl = __reduce_min_sync(gm, (ok && cnt == maxc) ? lab : kFull);
        if (vin && k == 0) {
          const uint32_t nl = dv ? bestl : oldv;
          c.lab_out[nodev] = nl;
          my_changed += (nl != oldv);
        }
      }
    } else {
      // one vertex per round
      for (uint32_t j = lo; j < hi; j++) {
        const uint32_t dv = __shfl_sync(kFull, d, j);
        const uint32_t bv = __shfl_sync(kFull, base, j);
        const uint32_t nodev = __shfl_sync(kFull, node, j);
        const uint32_t oldv = __shfl_sync(kFull, old, j);
        uint32_t bestl;
        if (dv <= 32) {
          const bool ok = lane < dv;
          const uint32_t lab = ok ? stage[bv + lane] : kFull;
          const uint32_t cnt = group_counts(ok, lab, kFull, 0u);
          const uint32_t maxc = __reduce_max_sync(kFull, cnt);
          bestl = __reduce_min_sync(kFull, (ok && cnt == maxc) ? lab : kFull);
        } else {
          // epoch table: no clearing, running argmax from the returned counts
          if (++epoch >= kLightEpochs) {
            for (uint32_t i = lane; i < kWarpSlots; i += 32) slots[i] = 0ull;
            __syncwarp();
            epoch = 1;
          }
          const EpochTable et{slots, min(next_pow2(2 * dv), kWarpSlots), epoch};  // cap > dv: every label fits
          uint64_t bp = 0;
          const auto ins = [&](uint32_t lab, uint32_t w) {
            const uint64_t cand = pack_best(et.insert(lab, w), lab);
            bp = cand > bp ? cand : bp;
          };
          // a step of one label extends the current run (fixed plan at R-MAT
          // scale 24: 13.48 -> 13.21 ms per iteration)
          WarpRun run;
          for (uint32_t k0 = 0; k0 < dv; k0 += 32) {
            const uint32_t k = k0 + lane;
            const bool ok = k < dv;
            const uint32_t lab = ok ? stage[bv + k] : kFull;
            if (run.extend(ok, lab)) continue;
            if (run.cnt && lane == 0) ins(run.lab, run.cnt);
            run.restart(ok, lab);
            const uint32_t w = warp_merge(ok, lab);
            if (w) ins(lab, w);
          }
          if (run.cnt && lane == 0) ins(run.lab, run.cnt);
          bestl = best_label(warp_max_u64(bp));
          __syncwarp();
        }
        if (lane == 0) {
          const uint32_t nl = dv ? bestl : oldv;
          c.lab_out[nodev] = nl;
          my_changed += (nl != oldv);
        }
      }
    }
    __syncwarp();
    src_skip += total;
    done |= batch;
  }
  changed += my_changed;
  if (a.seg_changed) {
    const uint32_t s = __reduce_add_sync(kFull, my_changed);
    if (lane == 0 && s) atomicAdd(a.seg_changed + seg, s);
  }
}

// The block variant over one plan segment.  A vertex that one warp's table
// and staging area hold (exact, degree <= kV1MaxDeg) is decoded and counted
// by one warp, eight of them side by side: its 256-bit segments number at
// most 64, so one vertex per block would leave most of the block idle while
// a few lanes decode.  A hub (larger, or at the sketch threshold) takes the
// whole block, whose 256 threads then decode its segments in parallel.
__device__ void block_segment(const IterArgs &a, const Ctx &c, BlockSh &sh, uint32_t *stage, uint32_t *tab,
                              uint32_t *wstage, unsigned long long *wslots, uint32_t &wepoch, uint32_t s,
                              const Seg sg, bool from_scratch, unsigned long long &changed) {
  const DevGraph &g = a.g;
  const uint32_t t = threadIdx.x, warp = t >> 5;
  bool fits = true;
  for (uint32_t p = sg.begin + t; p < sg.end; p += kThreads) {
    const uint32_t d = g.deg[p];
    fits &= d <= kV1MaxDeg && !(a.cms_thr != 0 && d >= a.cms_thr);
  }
  if (__syncthreads_and(fits)) {
    const int v = from_scratch ? kVarTwoPass : kVarWarp;
    for (uint32_t p = sg.begin + warp; p < sg.end; p += kWarps) light_chunk(a, c, wstage, wslots, wepoch, s, p, p + 1, v, changed);
    __syncthreads();  // the block's shared memory is free for the next item
    return;
  }
  for (uint32_t p = sg.begin; p < sg.end; p++) heavy_vertex(a, c, sh, stage, tab, s, p, from_scratch, changed);
}

}  // namespace

// Widens the kernel's busy span in a.ktime by this warp's start or end.
__device__ __forceinline__ void busy_mark(const IterArgs &a, int kernel, bool end) {
  if (a.ktime && (threadIdx.x & 31u) == 0) {
    const unsigned long long t = global_ns();
    if (end) atomicMax(a.ktime + kBusyKernels + kernel, t);
    else atomicMin(a.ktime + kernel, t);
  }
}

__global__ void __launch_bounds__(kThreads, 2) k_iterate(IterArgs a) {
  extern __shared__ uint32_t smem[];
  __shared__ BlockSh sh;
  uint32_t *stage = smem;         // kStage words
  uint32_t *tab = smem + kStage;  // kTableSlots keys + kTableSlots counts (or the sketch)
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  for (uint32_t i = t; i < 2 * kTableSlots; i += kThreads) tab[i] = 0u;
  if (t == 0) sh.hepoch = kHeavyEpochFirst;
  __syncthreads();
  const Ctx c = resolve(a);
  busy_mark(a, 2, false);
  unsigned long long changed = 0;
  uint32_t *qctr = a.work + kWorkCounters * (a.it_dev ? c.it : 0u) + kWqHeavy;

  // per-warp staging and exact table of the warp-scope paths
  unsigned long long *wslots = reinterpret_cast<unsigned long long *>(tab) + warp * kWarpSlots;
  uint32_t *wstage = stage + warp * kWarpStage;
  uint32_t wepoch = 0;

  // heavy items: one segment per block (largest first).  The next item is
  // claimed before the current one runs and its bits are prefetched into L2.
  if (t == 0) {
    const uint32_t i0 = atomicAdd(qctr, 1u);
    sh.item = i0;
    if (i0 < a.n_heavy) prefetch_l2(reinterpret_cast<const void *>(a.heavy[i0].pf_addr), a.heavy[i0].pf_bytes);
  }
  __syncthreads();
  uint32_t next = sh.item;
  for (;;) {
    const uint32_t i = next;
    __syncthreads();
    if (i >= a.n_heavy) break;
    if (t == 0) {
      const uint32_t in = atomicAdd(qctr, 1u);
      sh.item = in;
      if (in < a.n_heavy) prefetch_l2(reinterpret_cast<const void *>(a.heavy[in].pf_addr), a.heavy[in].pf_bytes);
    }
    __syncthreads();
    next = sh.item;
    const uint32_t s = a.heavy[i].tag;
    const bool from_scratch = a.seg_var[s] == kVarTwoPass;
    const Seg sg = a.segs[s];
    const long long t0 = clock64();
    block_segment(a, c, sh, stage, tab, wstage, wslots, wepoch, s, sg, from_scratch, changed);
    if (a.seg_cycles && t == 0)
      atomicAdd(reinterpret_cast<unsigned long long *>(a.seg_cycles + s),
                (unsigned long long)((clock64() - t0) * kWarps * a.cw_iterate));
  }

  // light chunks: a warp claims 4 consecutive chunks at a time, prefetches
  // the last 3 into L2 at once and runs them in order
  for (;;) {
    uint32_t i0 = 0;
    if (lane == 0) i0 = atomicAdd(qctr + 1, 4u);
    i0 = __shfl_sync(kFull, i0, 0);
    if (i0 >= a.n_light) break;
    WorkItem wi{};
    if (lane < 4 && i0 + lane < a.n_light) wi = a.light[i0 + lane];
    if (lane >= 1 && lane < 4 && i0 + lane < a.n_light)
      prefetch_l2(reinterpret_cast<const void *>(wi.pf_addr), wi.pf_bytes);
    for (uint32_t k = 0; k < 4 && i0 + k < a.n_light; k++) {
      const uint32_t item = __shfl_sync(kFull, wi.tag, k);
      const uint32_t s = item >> 3;
      const Seg sg = a.segs[s];
      const uint32_t p0 = sg.begin + (item & 7u) * 32u;
      const long long t0 = clock64();
      light_chunk(a, c, wstage, wslots, wepoch, s, p0, min(sg.end, p0 + 32u), a.seg_var[s], changed);
      if (a.seg_cycles && lane == 0)
        atomicAdd(reinterpret_cast<unsigned long long *>(a.seg_cycles + s),
                  (unsigned long long)((clock64() - t0) * a.cw_iterate));
    }
  }
  busy_mark(a, 2, true);
  flush_changed(c.changed, changed);
}

__device__ __forceinline__ uint32_t packed_vertex(const IterArgs &a, const Ctx &c, uint32_t p, uint32_t *lab);

// Many graphs, one persistent launch.  A ring queue holds (graph,
// iteration, segment) items; iteration 0 of every graph is queued by the
// host.  The block that finishes the last item of a graph's iteration reads
// that iteration's changed count and either retires the graph or queues all
// its segments for the next iteration, so an item never waits on another
// item.  Blocks wait (bounded) only on an empty queue slot.  Labels change
// during the launch, so they are read through L2.
__global__ void __launch_bounds__(kThreads, 2) k_batch(BatchArgs b) {
  extern __shared__ uint32_t smem[];
  __shared__ BlockSh sh;
  __shared__ IterArgs ia;
  __shared__ unsigned long long s_item, s_enq_base;
  __shared__ uint32_t s_last, s_enq;
  uint32_t *stage = smem;
  uint32_t *tab = smem + kStage;
  const uint32_t t = threadIdx.x, warp = t >> 5;
  for (uint32_t i = t; i < 2 * kTableSlots; i += kThreads) tab[i] = 0u;
  if (t == 0) sh.hepoch = kHeavyEpochFirst;
  __syncthreads();
  unsigned long long *wslots = reinterpret_cast<unsigned long long *>(tab) + warp * kWarpSlots;
  uint32_t *wstage = stage + warp * kWarpStage;
  uint32_t wepoch = 0;
  for (;;) {
    if (t == 0) {
      const unsigned long long idx = atomicAdd(b.head, 1ull);
      volatile unsigned long long *slot = b.queue + (idx % b.cap);
      unsigned long long e = *slot;
      unsigned long long spins = 0;
      while (e == kQueueEmpty) {
        if (*reinterpret_cast<volatile uint32_t *>(b.active) == 0u) break;
        if (++spins > b.spin_limit) {
          set_error(b.err, kErrTimeout);
          break;
        }
        __nanosleep(200);
        e = *slot;
      }
      if (e != kQueueEmpty) *slot = kQueueEmpty;
      __threadfence();
      s_item = e;
    }
    __syncthreads();
    const unsigned long long e = s_item;
    if (e == kQueueEmpty) break;
    const uint32_t gi = uint32_t(e >> 44), it = uint32_t(e >> 32) & 0xFFFu, s = uint32_t(e);
    if (t == 0) {
      const BatchGraph &bg = b.graphs[gi];
      ia = IterArgs{};  // every field this launch does not use is zero (null): no hub spill, no scratch
      ia.g = bg.g;
      ia.labs0 = bg.labs0;
      ia.labs1 = bg.labs1;
      ia.parity0 = 0;
      ia.it_dev = nullptr;
      ia.changed = b.changed + gi;
      ia.work = nullptr;
      ia.err = b.err;
      ia.segs = bg.segs;
      ia.seg_var = bg.seg_var;
      ia.seg_cycles = nullptr;
      ia.seg_changed = nullptr;
      ia.cms_thr = b.cms_thr;
      for (int r = 0; r < kCmsDepth; r++) ia.seeds[r] = b.seeds[r];
      ia.scratch = nullptr;
      ia.arc_off = nullptr;
      ia.scratch_labels = 0;
      ia.groups = nullptr;
      ia.n_groups = 0;
      ia.pidx = nullptr;
      ia.cursor = nullptr;
      ia.ktime = nullptr;
      ia.packed = nullptr;
      ia.n_packed = 0;
      ia.gtab = b.gtab;
      ia.gtab_slots = b.gtab_slots;
      ia.gbase = nullptr;  // every graph has its own labels
      ia.n_gbase = 0;
    }
    __syncthreads();
    Ctx c;
    c.it = it;
    c.lab_in = (it & 1u) ? ia.labs1 : ia.labs0;
    c.lab_out = (it & 1u) ? ia.labs0 : ia.labs1;
    c.changed = ia.changed;
    c.coherent = true;
    unsigned long long changed = 0;
    const Seg sg = ia.segs[s];
    const int v = ia.seg_var[s];
    if (v == kVarBlock || v == kVarTwoPass) {
      block_segment(ia, c, sh, stage, tab, wstage, wslots, wepoch, s, sg, false, changed);
    } else if (v == kVarPackedLanes) {
      // a tiny segment: one thread per position (<= 256 positions)
      if (sg.begin + t < sg.end) changed += packed_vertex(ia, c, sg.begin + t, stage + t * kPackedMaxDeg);
    } else {
      const uint32_t p0 = sg.begin + warp * 32u;  // light segments hold at most 8 chunks
      if (p0 < sg.end) light_chunk(ia, c, wstage, wslots, wepoch, s, p0, min(sg.end, p0 + 32u), v, changed);
    }
    flush_changed(c.changed, changed);
    __threadfence();
    __syncthreads();
    if (t == 0) {
      const uint32_t nseg = b.graphs[gi].nseg;
      s_last = (atomicAdd(b.done_items + gi, 1u) + 1u == nseg) ? 1u : 0u;
      s_enq = 0;
      if (s_last) {
        __threadfence();
        const unsigned long long ch = atomicExch(b.changed + gi, 0ull);
        b.done_items[gi] = 0;
        b.iters[gi] = it + 1;
        const bool stop = (b.early_exit && ch == 0ull) || it + 1 >= b.max_iter;
        if (stop) {
          __threadfence();
          atomicSub(b.active, 1u);
        } else {
          s_enq_base = atomicAdd(b.tail, (unsigned long long)nseg);
          s_enq = nseg;
        }
      }
    }
    __syncthreads();
    if (s_enq) {
      const unsigned long long tag = (uint64_t(gi) << 44) | (uint64_t(it + 1) << 32);
      for (uint32_t k = t; k < s_enq; k += kThreads) {
        __threadfence();
        b.queue[(s_enq_base + k) % b.cap] = tag | k;
      }
    }
    __syncthreads();
  }
}

__global__ void k_batch_init(const BatchGraph *graphs, uint32_t ngraphs) {
  for (uint32_t gi = blockIdx.x; gi < ngraphs; gi += gridDim.x) {
    const BatchGraph &bg = graphs[gi];
    for (uint64_t v = threadIdx.x; v < bg.g.n; v += blockDim.x) {
      bg.labs0[v] = uint32_t(v);
      bg.labs1[v] = uint32_t(v);
    }
  }
}

// One vertex of degree <= kPackedMaxDeg by one thread: it walks the vertex's
// whole bit range (or its small-CSR list), gathering each label as soon as
// its id is decoded, then takes the most frequent of its labels (smallest on
// ties) by pairwise counts.  Returns 1 when the label changed.
// lab: this thread's kPackedMaxDeg label slots (shared memory in k_packed,
// where a lane's slots start kPackedMaxDeg words after the previous lane's:
// an odd stride, so the 32 lanes' k-th slots fall in 32 different banks).
__device__ __forceinline__ uint32_t packed_vertex(const IterArgs &a, const Ctx &c, uint32_t p, uint32_t *lab) {
  const DevGraph &g = a.g;
  const uint32_t node = g.vertices[p];
  const uint32_t d = g.deg[p];
  const uint32_t old = ld_label(c, node);
  uint32_t k = 0;
  bool bad = d > kPackedMaxDeg;
  if (!bad && p < g.n_c) {
    // the walk stages the ids, then every label load is in flight at once (a
    // load in the walk's loop held the lane at its store: road grid 1404^2,
    // k_packed 0.096 -> 0.079 ms)
    const int64_t r = walk_vertex_buf<true>(g.words, g.offsets[p], g.offsets[p + 1], node, g.n, [&](uint32_t id) {
      if (k < kPackedMaxDeg) lab[k] = id;
      k++;
    });
    bad = r != int64_t(d);
    if (!bad) {
      uint32_t lv[kPackedMaxDeg];
#pragma unroll
      for (uint32_t j = 0; j < kPackedMaxDeg; j++) lv[j] = j < d ? ld_label(c, lab[j]) : 0u;
#pragma unroll
      for (uint32_t j = 0; j < kPackedMaxDeg; j++)
        if (j < d) lab[j] = lv[j];
    }
  } else if (!bad) {
    const uint32_t *ids = g.small_nbr + g.small_off[p - g.n_c];
    for (; k < d; k++) lab[k] = ld_label(c, ids[k]);
  }
  if (bad) {
    set_error(a.err, kErrBadStream);
    return 0;
  }
  if (d == 0) return 0;
  uint64_t best = 0;
  for (uint32_t x = 0; x < d; x++) {
    uint32_t cnt = 0;
    for (uint32_t y = 0; y < d; y++) cnt += lab[y] == lab[x];
    const uint64_t cand = pack_best(cnt, lab[x]);
    best = cand > best ? cand : best;
  }
  const uint32_t nl = best_label(best);
  c.lab_out[node] = nl;
  return nl != old;
}

// V2 (several vertices per warp) at its limit for the tiny bucket: one lane
// per position (packed_vertex), 32 vertices per warp.  No shared memory, no
// warp-wide steps.
__global__ void __launch_bounds__(kThreads) k_packed(IterArgs a) {
  // per thread kPackedMaxDeg label slots: a per-thread array indexed at run
  // time would live in local memory
  __shared__ uint32_t slab[kThreads * kPackedMaxDeg];
  const Ctx c = resolve(a);
  busy_mark(a, 3, false);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  unsigned long long changed = 0;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < a.n_packed; i += nw) {
    const long long t0 = clock64();
    const PackedChunk ch = a.packed[i];
    const uint32_t mine = lane < ch.np ? packed_vertex(a, c, ch.p0 + lane, slab + threadIdx.x * kPackedMaxDeg) : 0u;
    changed += mine;
    const uint32_t sc = __reduce_add_sync(kFull, mine);
    if (lane == 0) {
      if (a.seg_changed && sc) atomicAdd(a.seg_changed + ch.seg, sc);
      if (a.seg_cycles)
        atomicAdd(reinterpret_cast<unsigned long long *>(a.seg_cycles + ch.seg),
                  (unsigned long long)((clock64() - t0) * a.cw_packed));
    }
  }
  busy_mark(a, 3, true);
  flush_changed(c.changed, changed);
}

// Two-pass variant, pass 1.  Every 256-bit segment of the two-pass positions
// is decoded by one lane, which writes the labels of its ids (not the ids) to
// the scratch, so pass 2 only counts.  A warp takes one decode group (32
// segments) at a time from the iteration's work queue (IterArgs::work slot
// kWqGroups, zeroed before the launch).  Lane l finds its position with a warp scan of the positions'
// segment counts and a 5-step search; the lanes of one position reserve their
// output range with one atomicAdd on the position's cursor, since the labels
// of a position may sit in any order.  No block barriers: warps run alone.
// kGather (lpa_tune.gather_cache) picks the cache path of the residual label
// reads: 1 all through L2 only (ld.global.cg), leaving L1 to the bitstream;
// 2 all through L1, which pays when a few hot labels take many of the reads;
// 0 the labels of the lowest kHotIds ids (BFS order puts the hubs there)
// through L1 and the rest through L2 only.  A hot set about the size of the
// L1 left beside the window wins: against the lowest n/64 ids (262,144 at
// R-MAT scale 24) 8192 took the pre-pass from 2.336 to 2.257 ms at scale 24
// and the copy-model iteration from 24.75 to 24.34 ms, scale 22 within
// 0.5 %; 4096 and 16384 measured the same as 8192 at scale 24.
//
// kStage (lpa_tune.stage_stream) moves each group's stream span (the words its
// segments read, DecodeGroup::w0/wn) ahead of its decode with the copy
// engine: 1 a bulk prefetch of the next group's span into L2
// (cp.async.bulk.prefetch.L2) while the warp decodes the current one; 2 a 1-D
// bulk copy of the next group's span into one of two shared-memory buffers of
// the warp (cp.async.bulk ... mbarrier::complete_tx, 16-byte aligned, no
// multicast), completed on that buffer's mbarrier with a bounded wait, so the
// copy of group k + 1 overlaps the decode of group k; the lanes then read
// their words from the buffer (words outside the copied span, if any, from
// the stream itself).
//
// kPack (n <= 2^27, unstaged forms): a staged id carries its lane in its top
// 5 bits, so the window needs no owner bytes (one shared store per id fewer:
// pre-pass 2.45 -> 2.39 ms at R-MAT scale 24).
template <int kGather, int kStage, bool kPack>
__global__ void __launch_bounds__(kThreads, 4) k_decode_two_pass(IterArgs a) {
  __shared__ uint32_t stage[kWarps * kDecodeWindow];
  __shared__ uint8_t owner[kPack ? 1 : kWarps * kDecodeWindow];
  extern __shared__ __align__(16) uint32_t sspan[];  // kStage 2: kSpanSmemBytes of dynamic shared memory
  __shared__ uint64_t sbar[kStage == 2 ? kWarps * 2 : 1];
  using WS = typename std::conditional<kStage == 2, StagedWords, GWords>::type;
  const DevGraph &g = a.g;
  const Ctx c = resolve(a);
  const uint32_t hot = uint32_t(min(g.n, uint64_t(kHotIds)));  // kGather 0: ids below read through L1
  // label reads through L2 keep their lines there ahead of the scratch, which
  // is written with streaming stores (read once, by the count pass):
  // 4.417 -> 4.396 ms per iteration at R-MAT scale 24
  const uint64_t keep_pol = l2_evict_last_policy();
  busy_mark(a, 0, false);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  // Decode groups come from the iteration's work queue, kGroupClaim at a
  // time, each warp's next claim made one ahead so that its atomic is off the
  // critical path.  A fixed grid-stride assignment left SMs idle for 28 % of
  // the kernel at R-MAT scale 22 (ncu: 0.66 ms of SM activity in a 0.92 ms
  // launch): groups whose interval segments expand thousands of ids finished
  // late on the warps that drew them.
  uint32_t *gctr = a.work + kWorkCounters * (a.it_dev ? c.it : 0u) + kWqGroups;
  const auto claim = [&]() {
    uint32_t x = 0;
    if (lane == 0) x = atomicAdd(gctr, kGroupClaim);
    return __shfl_sync(kFull, x, 0);
  };
  uint32_t gi = claim();
  uint32_t ahead = claim(), cend = gi + kGroupClaim;
  uint32_t *wspan = sspan + (kStage == 2 ? warp * 2 * kSpanWords : 0);
  uint64_t *wbar = sbar + (kStage == 2 ? warp * 2 : 0);
  uint32_t phase[2] = {0u, 0u};
  // the words [lo, lo + n) of group gi's span that buffer b receives
  const auto span_of = [&](const DecodeGroup &d, uint64_t &lo, uint32_t &n) {
    lo = d.w0 & ~uint64_t(3);
    const uint64_t hi = min(min(d.w0 + d.wn, a.wend), lo + kSpanWords);
    n = hi > lo ? uint32_t((hi - lo) & ~uint64_t(3)) : 0u;
  };
  const auto issue = [&](uint32_t gi, uint32_t b) {  // lane 0
    const DecodeGroup d = a.groups[gi];
    uint64_t lo;
    uint32_t n;
    span_of(d, lo, n);
    if (n) bulk_load(wspan + b * kSpanWords, g.words + lo, n * 4u, wbar + b);
    else asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(wbar + b)) : "memory");
  };
  if (kStage == 2) {
    if (lane == 0) {
      mbar_init(wbar, 1u);
      mbar_init(wbar + 1, 1u);
    }
    fence_mbar_init();
    __syncwarp();
    if (lane == 0 && gi < a.n_groups) issue(gi, 0u);
  }
  // the group after gi: the next of its claim, else the first of the claim
  // made ahead (which then becomes the current claim)
  const auto advance = [&]() {
    if (gi + 1u < cend) {
      gi++;
    } else {
      gi = ahead;
      cend = ahead + kGroupClaim;
      ahead = claim();
    }
  };
  for (uint32_t it = 0; gi < a.n_groups; it++, advance()) {
    const long long t0 = clock64();
    const DecodeGroup gd = a.groups[gi];
    const uint32_t b = it & 1u;
    const uint32_t gnext = gi + 1u < cend ? gi + 1u : ahead;
    WS src;
    if (kStage == 1) {
      if (lane == 0 && gnext < a.n_groups) {
        const DecodeGroup dn = a.groups[gnext];
        const uint64_t hi = min(dn.w0 + dn.wn, a.wend);
        if (hi > dn.w0) prefetch_l2(g.words + dn.w0, (hi - dn.w0) * 4);
      }
    }
    if constexpr (kStage == 2) {
      // the other buffer's last reader (the previous group) is done: it
      // receives the next group's span while this one is decoded
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0 && gnext < a.n_groups) issue(gnext, b ^ 1u);
      if (!__all_sync(kFull, mbar_wait(wbar + b, phase[b], kBulkWaitTries))) {
        if (lane == 0) set_error(a.err, kErrTimeout);
        // neither copy may still write the buffers when the warp leaves
        mbar_wait(wbar + b, phase[b], kBulkWaitTries);
        if (gnext < a.n_groups) mbar_wait(wbar + (b ^ 1u), phase[b ^ 1u], kBulkWaitTries);
        break;
      }
      phase[b] ^= 1u;
      uint64_t lo;
      uint32_t n;
      span_of(gd, lo, n);
      src = StagedWords{g.words, wspan + b * kSpanWords, lo, n};
    } else {
      src = GWords{g.words};
    }
    const uint32_t pk = gd.p0 + lane;
    uint4 ix = make_uint4(0u, 0u, 0u, 0u);
    if (pk < g.n_c) ix = a.pidx[pk];
    uint32_t ns = ix.z + ix.w;
    if (lane == 0) ns = ns > gd.j0 ? ns - gd.j0 : 0u;
    const uint32_t incl = warp_incl_scan(ns, lane);
    const uint32_t total = min(__shfl_sync(kFull, incl, 31), min(gd.nlanes, 32u));
    // owner: the number of positions whose segments all precede this lane
    uint32_t o = 0;
#pragma unroll
    for (uint32_t st = 16; st; st >>= 1) {
      const uint32_t v = __shfl_sync(kFull, incl, o + st - 1);
      if (v <= lane) o += st;
    }
    const uint32_t os = o & 31u;
    const uint32_t run0 = __shfl_sync(kFull, incl - ns, os);  // first lane of this position's run
    const uint32_t run1 = min(__shfl_sync(kFull, incl, os), total);
    const uint32_t ibr = __shfl_sync(kFull, ix.x, os), rbr = __shfl_sync(kFull, ix.y, os);
    const uint32_t nsi = __shfl_sync(kFull, ix.z, os);
    const bool act = lane < total;
    const uint32_t p = gd.p0 + os;
    const uint32_t jj = lane - run0 + (os == 0 ? gd.j0 : 0u);
    const bool itv = jj < nsi;
    bool bad = false;
    uint32_t cnt = 0, items = 0, node = 0;
    uint64_t q = 0, end = 0;
    BitReaderT<WS> r;
    if (act) {
      const uint64_t o0 = g.offsets[p];
      end = g.offsets[p + 1];
      node = g.vertices[p];
      q = o0 + (itv ? uint64_t(ibr) + uint64_t(kSegBits) * jj : uint64_t(rbr) + uint64_t(kSegBits) * (jj - nsi));
      if (q >= end) {
        bad = true;
      } else {
        r.seek(src, q);
        cnt = r.gamma(bad);
        if (!itv) {
          items = cnt;
        } else {
          for (uint32_t k = 0; k < cnt && !bad; k++) {
            r.gamma(bad);
            items += r.gamma(bad) + kMinItv;
            if (r.pos() > end) bad = true;
          }
        }
      }
      if (bad) {
        cnt = 0;
        items = 0;
      }
    }
    // output ranges: exclusive scan of items within the position's run
    const uint32_t iincl = warp_incl_scan(items, lane);
    const uint32_t run_before = __shfl_sync(kFull, iincl - items, run0 & 31u);
    const uint32_t run_total = __shfl_sync(kFull, iincl, (run1 - 1) & 31u) - run_before;
    uint32_t base = 0;
    if (act && lane == run0 && run_total) base = atomicAdd(a.cursor + p, run_total);
    base = __shfl_sync(kFull, base, run0 & 31u);
      // residual segments, in windows of kDecodeWindow items of the group:
    // each lane decodes its own segment's ids into the warp's staging area
    // (its lane number beside each), then the warp gathers the window's
    // labels with 8 loads per lane in flight and stores them, consecutive
    // ids of a position to consecutive addresses
    uint64_t obase = 0;  // scratch index of this lane's first item
    bool coop = false;   // an interval segment, expanded by the whole warp below
    uint32_t ritems = 0;
    if (act) {
      const uint32_t d = g.deg[p];
      const uint32_t off = base + (iincl - items) - run_before;
      obase = a.arc_off[p] + off;
      if (uint64_t(off) + items > d) bad = true;
      else if (items && itv) coop = true;
      else ritems = items;
    }
    const uint32_t rincl = warp_incl_scan(ritems, lane);
    const uint32_t rexcl = rincl - ritems;
    const uint32_t rtot = __shfl_sync(kFull, rincl, 31);
    // window item f of lane l goes to scratch[gb + drel_l + f] (32-bit
    // arithmetic) when the group's residual items lie within 2^32 of lane 0's
    // first, which holds the lowest scratch index of the group
    const uint64_t gb = (uint64_t(__shfl_sync(kFull, uint32_t(obase >> 32), 0)) << 32) |
                        __shfl_sync(kFull, uint32_t(obase), 0);
    const bool rel32 = __all_sync(kFull, ritems == 0u || ((obase + ritems - gb) >> 32) == 0ull);
    const uint32_t drel = uint32_t(obase - gb) - rexcl;
    const uint32_t nmax = uint32_t(g.n - 1);
    uint32_t *wst = stage + warp * kDecodeWindow;
    uint8_t *wown = owner + (kPack ? 0u : warp * kDecodeWindow);
    uint32_t done = 0, v = 0;
    for (uint32_t w0 = 0; w0 < rtot; w0 += kDecodeWindow) {
      const uint32_t w1 = min(w0 + kDecodeWindow, rtot);
      // this lane's items up to `lim` fall in this window, item i at window
      // index rexcl + i - w0 (>= 0 for every item not yet written)
      const uint32_t lim = rexcl + done < w1 ? min(ritems, w1 - rexcl) : done;
      uint32_t *dst = wst + (int32_t(rexcl) - int32_t(w0));
      // staged: the id with its lane in the top bits (kPack: the id's low 27
      // bits, so the lane stays intact) or in the owner bytes; the gather
      // clamps it to n - 1, once per 32 ids rather than once per code
      const auto put = [&](uint32_t k, uint32_t id) {
        if constexpr (kPack) {
          dst[k] = (id & 0x07FFFFFFu) | (lane << 27);
        } else {
          dst[k] = id;
          wown[int32_t(rexcl) - int32_t(w0) + int32_t(k)] = uint8_t(lane);
        }
      };
      if (done == 0 && lim > 0) {
        v = zigzag_first(node, r.zeta3(bad));
        put(0, v);
        done = 1;
      }
      for (; done < lim; done++) {
        v += r.zeta3(bad) + 1u;
        put(done, v);
      }
      // a segment's ids ascend, so its last one is its largest: an id past
      // n - 1 reads label n - 1, and the error word reports the stream (its
      // end is checked once, below).  Clamping instead of testing every id
      // took the pre-pass from 2.49 to 2.45 ms at R-MAT scale 24.
      if (done) bad |= v > nmax;
      __syncwarp();
      for (uint32_t f0 = w0; f0 < w1; f0 += 256) {
        uint32_t lv[8];
#pragma unroll
        for (int u = 0; u < 8; u++) {
          const uint32_t f = f0 + 32u * u + lane;
          const uint32_t id = f < w1 ? min(kPack ? wst[f - w0] & 0x07FFFFFFu : wst[f - w0], nmax) : 0u;
          lv[u] = f >= w1 ? 0u
                  : (kGather == 2 || (kGather == 0 && id < hot)) ? __ldg(c.lab_in + id)
                                                                  : ld_cg_keep(c.lab_in + id, keep_pol);
        }
        if (rel32) {
#pragma unroll
          for (int u = 0; u < 8; u++) {
            const uint32_t f = f0 + 32u * u + lane;
            const uint32_t ol = f < w1 ? (kPack ? wst[f - w0] >> 27 : wown[f - w0]) : 0u;
            const uint32_t rel = __shfl_sync(kFull, drel, ol) + f;
            if (f < w1) __stcs(a.scratch + gb + rel, lv[u]);
          }
        } else {
#pragma unroll
          for (int u = 0; u < 8; u++) {
            const uint32_t f = f0 + 32u * u + lane;
            const uint32_t ol = f < w1 ? (kPack ? wst[f - w0] >> 27 : wown[f - w0]) : 0u;
            const uint64_t ob = (uint64_t(__shfl_sync(kFull, uint32_t(obase >> 32), ol)) << 32) |
                                __shfl_sync(kFull, uint32_t(obase), ol);
            const uint32_t ox = __shfl_sync(kFull, rexcl, ol);
            if (f < w1) __stcs(a.scratch + ob + (f - ox), lv[u]);
          }
        }
      }
      __syncwarp();
    }
    if (ritems && r.pos() > end) bad = true;
    // interval segments: one (left, len) pair per lane per round, expanded by
    // the whole warp (an interval can hold thousands of ids).  A round with
    // few intervals copies them one after another, 32 consecutive ids per
    // step (a broadcast of the interval, then coalesced label loads and
    // stores); a round with many short ones expands their concatenation,
    // each lane taking every 32nd id and finding its interval by a search
    // over the lanes' scan.  The round takes the form with the lower
    // estimated instruction count: per interval 16 + 4 per 32 ids, against
    // 100 per 128 ids of the concatenation.  At R-MAT scale 24 (BFS order,
    // 2.5 % of compressed arcs in intervals) the one-at-a-time form took the
    // pre-pass from 3.14 to 2.93 ms.
    if (__any_sync(kFull, coop)) {
      uint32_t left_todo = 0, nextbase = 0, w = 0;
      if (coop) {
        r.seek(src, q);
        left_todo = r.gamma(bad);
      }
      // a section's last segment takes the overflow of the one before: < 512 bits, < 256 pairs
      for (uint32_t round = 0; round < 512u && __any_sync(kFull, coop && left_todo); round++) {
        uint32_t lo = 0, len = 0;
        if (coop && left_todo) {
          const uint32_t l = r.gamma(bad);
          lo = (left_todo == cnt) ? zigzag_first(node, l) : nextbase + l + 1u;
          len = r.gamma(bad) + kMinItv;
          left_todo--;
          if (bad || uint64_t(lo) + len > g.n || w + len > items) {
            bad = true;
            len = 0;
            left_todo = 0;
          }
          nextbase = lo + len;
        }
        const uint32_t incl2 = warp_incl_scan(len, lane);
        const uint32_t tot = __shfl_sync(kFull, incl2, 31);
        const uint64_t dst = obase + w;  // where this lane's interval goes
        const uint32_t solo = __reduce_add_sync(kFull, len ? 16u + 4u * ((len + 31u) >> 5) : 0u);
        if (solo <= 100u * ((tot + 127u) >> 7)) {
          for (uint32_t m = __ballot_sync(kFull, len != 0u); m; m &= m - 1u) {
            const uint32_t l = uint32_t(__ffs(m) - 1);
            const uint32_t lo_l = __shfl_sync(kFull, lo, l), len_l = __shfl_sync(kFull, len, l);
            const uint64_t d_l = (uint64_t(__shfl_sync(kFull, uint32_t(dst >> 32), l)) << 32) |
                                 __shfl_sync(kFull, uint32_t(dst), l);
            for (uint32_t k0 = 0; k0 < len_l; k0 += 128) {
              uint32_t lv[4];
#pragma unroll
              for (int u = 0; u < 4; u++) {
                const uint32_t k = k0 + 32u * u + lane;
                lv[u] = k < len_l ? ld_label(c, lo_l + k) : 0u;
              }
#pragma unroll
              for (int u = 0; u < 4; u++) {
                const uint32_t k = k0 + 32u * u + lane;
                if (k < len_l) __stcs(a.scratch + d_l + k, lv[u]);
              }
            }
          }
        } else {
          // 4 ids per lane per step, their loads in flight together
          for (uint32_t i0 = 0; i0 < tot; i0 += 128) {
            uint32_t lv[4];
            uint64_t at[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
              const uint32_t i = i0 + 32u * u + lane;
              uint32_t ow = 0;
#pragma unroll
              for (uint32_t st = 16; st; st >>= 1) {
                const uint32_t v = __shfl_sync(kFull, incl2, ow + st - 1);
                if (v <= i) ow += st;
              }
              ow &= 31u;
              const uint32_t first = __shfl_sync(kFull, incl2 - len, ow);
              const uint32_t olo = __shfl_sync(kFull, lo, ow);
              const uint64_t odst = (uint64_t(__shfl_sync(kFull, uint32_t(dst >> 32), ow)) << 32) |
                                    __shfl_sync(kFull, uint32_t(dst), ow);
              at[u] = odst + (i - first);
              lv[u] = i < tot ? ld_label(c, olo + (i - first)) : 0u;
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
              if (i0 + 32u * u + lane < tot) __stcs(a.scratch + at[u], lv[u]);
          }
        }
        w += len;
      }
      if (coop && (left_todo || w != items)) bad = true;
    }
    if (__any_sync(kFull, bad) && lane == 0) set_error(a.err, kErrBadStream);
    if (a.seg_cycles && lane == 0)
      atomicAdd(reinterpret_cast<unsigned long long *>(a.seg_cycles + gd.seg),
                (unsigned long long)((clock64() - t0) * a.cw_decode));
  }
  busy_mark(a, 0, true);
}

#define LPA_DECODE_FORMS(G)                                           \
  template __global__ void k_decode_two_pass<G, 0, false>(IterArgs a); \
  template __global__ void k_decode_two_pass<G, 1, false>(IterArgs a); \
  template __global__ void k_decode_two_pass<G, 2, false>(IterArgs a); \
  template __global__ void k_decode_two_pass<G, 0, true>(IterArgs a);
LPA_DECODE_FORMS(0)
LPA_DECODE_FORMS(1)
LPA_DECODE_FORMS(2)
#undef LPA_DECODE_FORMS

namespace {

// f(ok, label) for this warp's share of src[0..d): 32U-label blocks w,
// w + nw, ... with U loads per lane in flight; warp-synchronous.  keep: the
// labels will be read again soon (keep them in L2).
template <bool keep, int U = 8, class F>
__device__ __forceinline__ void warp_stream(const uint32_t *__restrict__ src, uint32_t d, uint32_t w, uint32_t nw,
                                            F &&f, const uint32_t *__restrict__ labels = nullptr) {
  const uint32_t lane = threadIdx.x & 31u;
  for (uint32_t b0 = w * 32u * U; b0 < d; b0 += nw * 32u * U) {
    uint32_t v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint32_t k = b0 + 32u * u + lane;
      v[u] = k < d ? (keep ? __ldcg(src + k) : __ldcs(src + k)) : 0u;
    }
    if (labels) {  // src holds ids: gather their labels
#pragma unroll
      for (int u = 0; u < U; u++)
        v[u] = (b0 + 32u * u + lane < d) ? (v[u] < kHotIds ? __ldg(labels + v[u]) : __ldcg(labels + v[u])) : 0u;
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const uint32_t k = b0 + 32u * u;
      if (k < d) f(k + lane < d, v[u]);
    }
  }
}

// Exact counts of this warp's share of src[0..d) (32U-label blocks) into et,
// with a running argmax in best (the count insert() returns is the label's
// total so far).
template <int U = 8>
__device__ __forceinline__ void count_exact(const EpochTable &et, const uint32_t *__restrict__ src, uint32_t d,
                                            uint32_t w, uint32_t nw, uint64_t &best,
                                            const uint32_t *__restrict__ labels = nullptr) {
  const uint32_t lane = threadIdx.x & 31u;
  const auto ins = [&](uint32_t lab, uint32_t c) {
    const uint64_t cand = pack_best(et.insert(lab, c), lab);
    best = cand > best ? cand : best;
  };
  WarpRun run;
  warp_stream<false, U>(src, d, w, nw, [&](bool ok, uint32_t lab) {
    if (run.extend(ok, lab)) return;
    if (run.cnt && lane == 0) ins(run.lab, run.cnt);
    run.restart(ok, lab);
    const uint32_t c = warp_merge(ok, lab);
    if (c) ins(lab, c);
  }, labels);
  if (run.cnt && lane == 0) ins(run.lab, run.cnt);
}

// The sketch of src[0..d) by the whole block in 32U-label blocks: every
// occurrence added to the zeroed counters cms (a warp-uniform run of one
// label adds once), then the running argmax of the estimate over the labels
// in best.  Lanes are not folded by label first (warp_merge): the shared
// memory atomics absorb the conflicts of a mixed step for less than the
// folding costs (count pass 2.55 -> 2.40 ms at R-MAT scale 24).
template <int U>
__device__ __forceinline__ void sketch_count(uint32_t *cms, const uint32_t *__restrict__ src, uint32_t d, uint32_t lb,
                                             const uint32_t *seeds, uint64_t &best) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const auto add = [&](uint32_t lab, uint32_t w) {
#pragma unroll
    for (int r = 0; r < kCmsDepth; r++)
      atomicAdd(&cms[r * kCmsWidth + (cm_hash(r, (lab - lb) ^ seeds[r]) & (kCmsWidth - 1))], w);
  };
  WarpRun run;
  warp_stream<true, U>(src, d, warp, kWarps, [&](bool ok, uint32_t lab) {
    if (run.extend(ok, lab)) return;
    if (run.cnt && lane == 0) add(run.lab, run.cnt);
    run.restart(ok, lab);
    if (ok) add(lab, 1u);
  });
  if (run.cnt && lane == 0) add(run.lab, run.cnt);
  __syncthreads();
  // the estimate depends on the label only: a step whose labels all equal
  // the label evaluated last adds nothing
  uint32_t seen = kFull;
  warp_stream<false, U>(src, d, warp, kWarps, [&](bool ok, uint32_t lab) {
    const uint32_t okm = __ballot_sync(kFull, ok);
    if (__ballot_sync(kFull, ok && lab == seen) == okm) return;
    seen = __shfl_sync(kFull, lab, __ffs(okm) - 1);
    if (ok) {
      uint32_t est = kFull;
#pragma unroll
      for (int r = 0; r < kCmsDepth; r++) {
        const uint32_t v = cms[r * kCmsWidth + (cm_hash(r, (lab - lb) ^ seeds[r]) & (kCmsWidth - 1))];
        est = v < est ? v : est;
      }
      const uint64_t cand = pack_best(est, lab);
      best = cand > best ? cand : best;
    }
  });
}

// Block-wide maximum of v, returned to every thread.
__device__ __forceinline__ uint64_t block_max_u64(uint64_t v, uint64_t *red) {
  v = warp_max_u64(v);
  if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  uint64_t m = 0;
#pragma unroll
  for (int w = 0; w < kWarps; w++) m = red[w] > m ? red[w] : m;
  __syncthreads();
  return m;
}

}  // namespace

// Two-pass variant, pass 2.  The labels of every compressed two-pass
// position sit in the scratch, so this kernel mostly streams and counts
// (positions of the small CSR gather their labels); it holds no staging area
// and runs five blocks per SM (48 registers).  Block items (largest first): exact
// degrees up to kCountBlockMax in a 4096-slot block table, or the sketch;
// the warps stream disjoint 256-label blocks of the vertex.  Warp items: up
// to 4 (tunable) positions of degree <= kCountWarpMax, one vertex at a time in the
// warp's 512-slot table, or up to 32 positions of degree <= 32 on G-lane
// groups.  The same shared memory serves the warp tables, the block table
// (block epochs, disjoint from the warps') and the sketch (cleared before and
// after use).  Every position's pre-pass cursor is reset here.
template <bool kBulk>
__global__ void __launch_bounds__(kThreads, 5) k_count_two_pass(IterArgs a) {
  extern __shared__ __align__(128) unsigned long long cslots[];
  __shared__ uint64_t red[kWarps];
  __shared__ uint64_t s_bar[kWarps];  // per warp: completion of its bulk copies
  __shared__ uint32_t s_has, s_epoch;
  __shared__ BlockItem s_bi;
  const DevGraph &g = a.g;
  const Ctx c = resolve(a);
  busy_mark(a, 1, false);
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  for (uint32_t i = t; i < kCountBlockSlots; i += kThreads) cslots[i] = 0ull;
  if (t == 0) s_epoch = kHeavyEpochFirst;
  if (lane == 0) mbar_init(s_bar + warp, 1u);
  fence_mbar_init();
  __syncthreads();
  uint32_t *qctr = a.work + kWorkCounters * (a.it_dev ? c.it : 0u) + kWqBlock;
  unsigned long long changed = 0;

  // Block items, claimed ahead: while the block works on item k, thread 0
  // holds item k + 1 (loaded) and the claim of item k + 2, so neither the
  // queue atomic nor the item load sits on an item's critical path.  An item
  // carries its position's degree, scratch offset and vertex id, so the
  // block streams labels at once.
  BlockItem nxt{};
  bool has_nxt = false;
  uint32_t claim = 0;
  if (t == 0) {
    const uint32_t c0 = atomicAdd(qctr, 1u), c1 = atomicAdd(qctr, 1u);
    s_has = c0 < a.n_cblock;
    if (s_has) s_bi = a.cblock[c0];
    has_nxt = c1 < a.n_cblock;
    if (has_nxt) nxt = a.cblock[c1];
    claim = atomicAdd(qctr, 1u);
    if (++s_epoch > 0xFFFFu) s_epoch = 0;
  }
  for (;;) {
    __syncthreads();
    if (!s_has) break;
    const BlockItem it = s_bi;
    if (s_epoch == 0) {  // the block epochs wrapped: clear the table once
      for (uint32_t k = t; k < kCountBlockSlots; k += kThreads) cslots[k] = 0ull;
      __syncthreads();
      if (t == 0) s_epoch = kHeavyEpochFirst;
    }
    __syncthreads();  // every thread holds the item before thread 0 moves on
    const long long t0 = clock64();
    const uint32_t d = it.d;
    const uint32_t *src = a.scratch + it.ao;
    uint32_t old = 0;
    if (t == 0) {
      a.cursor[it.p] = 0u;
      old = ld_label(c, it.node);  // needed at the end only
    }
    uint64_t best = 0;
    if (it.kind == kCountSketch) {
      uint32_t *cms = reinterpret_cast<uint32_t *>(cslots);
      for (uint32_t k = t; k < kCmsDepth * kCmsWidth; k += kThreads) cms[k] = 0u;
      const uint32_t lb = label_base(a, it.node);
      __syncthreads();
      sketch_count<8>(cms, src, d, lb, a.seeds, best);  // smaller blocks gain nothing at degree >= 1024
      best = block_max_u64(best, red);
      // leave no counter behind that a table could read as one of its slots
      for (uint32_t k = t; k < kCmsDepth * kCmsWidth; k += kThreads) cms[k] = 0u;
    } else {
      // blocks small enough that every warp takes one: the critical path of
      // a vertex of 512..1024 labels is one block of 64 or 128, not 256
      const EpochTable et{cslots, min(next_pow2(2 * d), kCountBlockSlots), s_epoch};
      if (d <= 32u * 2u * kWarps) count_exact<2>(et, src, d, warp, kWarps, best);
      else if (d <= 32u * 4u * kWarps) count_exact<4>(et, src, d, warp, kWarps, best);
      else count_exact<8>(et, src, d, warp, kWarps, best);
      best = block_max_u64(best, red);
    }
    if (t == 0) {
      const uint32_t nl = d ? best_label(best) : old;
      c.lab_out[it.node] = nl;
      changed += (nl != old);
      if (a.seg_changed && nl != old) atomicAdd(a.seg_changed + it.seg, 1u);
      if (a.seg_cycles)
        atomicAdd(reinterpret_cast<unsigned long long *>(a.seg_cycles + it.seg),
                  (unsigned long long)((clock64() - t0) * kWarps * a.cw_count));
      // advance the pipeline (the block reads s_bi after the loop-top barrier)
      s_has = has_nxt;
      s_bi = nxt;
      has_nxt = claim < a.n_cblock;
      if (has_nxt) nxt = a.cblock[claim];
      claim = atomicAdd(qctr, 1u);
      if (++s_epoch > 0xFFFFu) s_epoch = 0;
    }
  }

  unsigned long long *wslots = cslots + warp * kCountWarpSlots;
  uint32_t wepoch = 0;
  uint32_t bphase = 0;  // parity of this warp's next bulk-copy phase
  bool stop = false;    // a bulk copy did not complete in time
  while (!stop) {
    uint32_t i0 = 0;
    const uint32_t claim = a.warp_claim ? a.warp_claim : 2u;
    if (lane == 0) i0 = atomicAdd(qctr + 1, claim);
    i0 = __shfl_sync(kFull, i0, 0);
    if (i0 >= a.n_cwarp) break;
    for (uint32_t q = i0; q < i0 + claim && q < a.n_cwarp; q++) {
      const CountItem it = a.cwarp[q];
      const long long t0 = clock64();
      uint32_t my_changed = 0;
      if (it.kind == kCountGroups) {
        const uint32_t p = it.p0 + lane;
        const bool valid = lane < it.np;
        const uint32_t node = valid ? g.vertices[p] : 0u;
        const uint32_t d = valid ? g.deg[p] : 0u;
        const uint32_t old = valid ? ld_label(c, node) : 0u;
        // compressed positions: labels in the scratch; the small CSR: ids
        const bool ids = it.p0 >= g.n_c;
        const uint64_t ao = !valid ? 0ull : (ids ? uint64_t(g.small_off[p - g.n_c]) : a.arc_off[p]);
        if (valid && !ids) a.cursor[p] = 0u;
        // the positions are consecutive, so their neighbours are one range:
        // stage all its labels in the warp's table memory first (8 loads per
        // lane in flight), then count from shared memory
        const uint32_t incl = warp_incl_scan(d, lane);
        const uint32_t excl = incl - d;
        const uint32_t total = __shfl_sync(kFull, incl, 31);  // <= 32 * 32
        const uint64_t ao0 = (uint64_t(__shfl_sync(kFull, uint32_t(ao >> 32), 0)) << 32) |
                             __shfl_sync(kFull, uint32_t(ao), 0);
        uint32_t *wstage = reinterpret_cast<uint32_t *>(wslots);
        // scratch labels: one bulk copy of the 16-byte-aligned bytes around
        // the range (the scratch is padded at its end), the labels then at
        // wstage[sh0..); the small CSR gathers ids
        const uint64_t b_lo = (ao0 * 4u) & ~15ull, b_hi = ((ao0 + total) * 4u + 15u) & ~15ull;
        const bool bulk = kBulk && !ids && total >= kBulkMinLabels && b_hi - b_lo <= kCountWarpSlots * 8u;
        const uint32_t sh0 = bulk ? uint32_t(ao0 & 3u) : 0u;
        if (bulk) {
          fence_proxy_async_smem();  // this lane's earlier accesses to wstage come first
          __syncwarp();
          if (lane == 0)
            bulk_load(wstage, reinterpret_cast<const char *>(a.scratch) + b_lo, uint32_t(b_hi - b_lo), s_bar + warp);
          if (!__all_sync(kFull, mbar_wait(s_bar + warp, bphase, kBulkWaitTries))) {
            if (lane == 0) set_error(a.err, kErrTimeout);
            mbar_wait(s_bar + warp, bphase, kBulkWaitTries);  // the copy still writes wstage
            stop = true;
            break;
          }
          bphase ^= 1u;
        } else {
          for (uint32_t k0 = 0; k0 < total; k0 += 256) {
            uint32_t v[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
              const uint32_t kk = k0 + 32u * u + lane;
              v[u] = kk >= total ? 0u : (ids ? __ldg(g.small_nbr + ao0 + kk) : __ldcs(a.scratch + ao0 + kk));
            }
            if (ids) {
#pragma unroll
              for (int u = 0; u < 8; u++) v[u] = (k0 + 32u * u + lane < total) ? ld_label_gather(c, v[u]) : 0u;
            }
#pragma unroll
            for (int u = 0; u < 8; u++)
              if (k0 + 32u * u + lane < total) wstage[k0 + 32u * u + lane] = v[u];
          }
        }
        __syncwarp();
        const uint32_t *lbl = wstage + sh0;
        // a vertex whose labels are all equal takes that label: lane v checks
        // its own vertex; only the others are counted below
        bool mixed = false;
        const uint32_t first = (lane < it.np && d) ? lbl[excl] : 0u;
        for (uint32_t j = 1; j < d; j++) mixed |= lbl[excl + j] != first;
        if (lane < it.np && d && !mixed) {  // an isolated vertex keeps its label in both buffers
          c.lab_out[node] = first;
          my_changed += (first != old);
        }
        const uint32_t rest = __ballot_sync(kFull, mixed);
        if (rest) {
          // G-lane groups over the mixed vertices, 32 / G of them a round
          const uint32_t nrest = __popc(rest);
          const uint32_t dmax = __reduce_max_sync(kFull, mixed ? d : 0u);
          const uint32_t G = next_pow2(dmax);
          const uint32_t per = 32 / G;
          const uint32_t gl = lane / G, k = lane % G;
          const uint32_t gm = (G == 32) ? kFull : (((1u << G) - 1u) << (gl * G));
          for (uint32_t v0 = 0; v0 < nrest; v0 += per) {
            const bool vin = v0 + gl < nrest;
            const uint32_t srcl = vin ? __fns(rest, 0, v0 + gl + 1) : 0u;
            const uint32_t dv = __shfl_sync(kFull, d, srcl);
            const uint32_t nodev = __shfl_sync(kFull, node, srcl);
            const uint32_t oldv = __shfl_sync(kFull, old, srcl);
            const uint32_t ev = __shfl_sync(kFull, excl, srcl);
            const bool ok = vin && k < dv;
            const uint32_t lab = ok ? lbl[ev + k] : kFull;
            const uint32_t cnt = group_counts(ok, lab, gm, gl);
            const uint32_t maxc = __reduce_max_sync(gm, cnt);
            const uint32_t bestl = __reduce_min_sync(gm, (ok && cnt == maxc) ? lab : kFull);
            if (vin && k == 0) {
              c.lab_out[nodev] = bestl;
              my_changed += (bestl != oldv);
            }
          }
        }
        __syncwarp();
        // the staged labels must not read as table slots later
        const uint32_t used = bulk ? uint32_t(b_hi - b_lo) / 8u : (total + 1) / 2;
        for (uint32_t k2 = lane; k2 < used; k2 += 32) wslots[k2] = 0ull;
        __syncwarp();
      } else {
        // every vertex's metadata in one round of loads (lane j: vertex j)
        const bool vj = lane < it.np;
        const uint32_t nodej = vj ? g.vertices[it.p0 + lane] : 0u;
        const uint32_t dj = vj ? g.deg[it.p0 + lane] : 0u;
        const uint32_t oldj = vj ? ld_label(c, nodej) : 0u;
        for (uint32_t j = 0; j < it.np; j++) {
          const uint32_t p = it.p0 + j;
          const uint32_t node = __shfl_sync(kFull, nodej, j);
          const uint32_t d = __shfl_sync(kFull, dj, j);
          const uint32_t old = __shfl_sync(kFull, oldj, j);
          const bool ids = p >= g.n_c;
          if (lane == 0 && !ids) a.cursor[p] = 0u;
          if (++wepoch >= kLightEpochs) {
            for (uint32_t k = lane; k < kCountWarpSlots; k += 32) wslots[k] = 0ull;
            __syncwarp();
            wepoch = 1;
          }
          const EpochTable et{wslots, min(next_pow2(2 * d), kCountWarpSlots), wepoch};
          uint64_t bp = 0;
          if (ids) count_exact(et, g.small_nbr + g.small_off[p - g.n_c], d, 0, 1, bp, c.lab_in);
          // a vertex of at most 128 labels loads them in one step of four rows
          // rather than eight (count pass 2.26 -> 2.21 ms at R-MAT scale 24)
          else if (d <= 128) count_exact<4>(et, a.scratch + a.arc_off[p], d, 0, 1, bp);
          else count_exact(et, a.scratch + a.arc_off[p], d, 0, 1, bp);
          bp = warp_max_u64(bp);
          if (lane == 0) {
            const uint32_t nl = d ? best_label(bp) : old;
            c.lab_out[node] = nl;
            my_changed += (nl != old);
          }
          __syncwarp();
        }
      }
      changed += my_changed;
      const uint32_t sc = __reduce_add_sync(kFull, my_changed);
      if (lane == 0) {
        if (a.seg_changed && sc) atomicAdd(a.seg_changed + it.seg, sc);
        if (a.seg_cycles)
          atomicAdd(reinterpret_cast<unsigned long long *>(a.seg_cycles + it.seg),
                    (unsigned long long)((clock64() - t0) * a.cw_count));
      }
    }
  }
  busy_mark(a, 1, true);
  flush_changed(c.changed, changed);
}

template __global__ void k_count_two_pass<false>(IterArgs a);
template __global__ void k_count_two_pass<true>(IterArgs a);

template <int G>
static void launch_decode_form(uint32_t stage, int grid, cudaStream_t s, const IterArgs &a) {
  if (stage == 1) k_decode_two_pass<G, 1, false><<<grid, kThreads, 0, s>>>(a);
  else if (stage == 2) k_decode_two_pass<G, 2, false><<<grid, kThreads, kSpanSmemBytes, s>>>(a);
  else if (a.g.n <= (1ull << 27)) k_decode_two_pass<G, 0, true><<<grid, kThreads, 0, s>>>(a);
  else k_decode_two_pass<G, 0, false><<<grid, kThreads, 0, s>>>(a);
}

cudaError_t prepare_decode_two_pass() {
  cudaError_t e = cudaFuncSetAttribute(k_decode_two_pass<0, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       int(kSpanSmemBytes));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_decode_two_pass<1, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSpanSmemBytes));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_decode_two_pass<2, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSpanSmemBytes));
  return e;
}

void launch_decode_two_pass(uint32_t gather_cache, uint32_t stage, int grid, cudaStream_t s, const IterArgs &a) {
  if (gather_cache == 1) launch_decode_form<1>(stage, grid, s, a);
  else if (gather_cache == 2) launch_decode_form<2>(stage, grid, s, a);
  else launch_decode_form<0>(stage, grid, s, a);
}

void launch_count_two_pass(bool bulk, int grid, cudaStream_t s, const IterArgs &a) {
  if (bulk) k_count_two_pass<true><<<grid, kThreads, kCountSmemBytes, s>>>(a);
  else k_count_two_pass<false><<<grid, kThreads, kCountSmemBytes, s>>>(a);
}

cudaError_t occupancy_decode_two_pass(int *blocks) {
  // the forms without shared-memory staging (the default); the staged form
  // holds more shared memory and runs fewer blocks per SM
  int b0 = 1, b1 = 1, b2 = 1;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_decode_two_pass<0, 0, false>, kThreads, 0);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_decode_two_pass<1, 0, false>, kThreads, 0);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b2, k_decode_two_pass<2, 0, false>, kThreads, 0);
  *blocks = b0 < b1 ? (b0 < b2 ? b0 : b2) : (b1 < b2 ? b1 : b2);
  return e;
}

cudaError_t occupancy_count_two_pass(int *blocks) {
  int b0 = 1, b1 = 1;
  cudaError_t e =
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b0, k_count_two_pass<false>, kThreads, kCountSmemBytes);
  if (e == cudaSuccess)
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b1, k_count_two_pass<true>, kThreads, kCountSmemBytes);
  *blocks = b0 < b1 ? b0 : b1;
  return e;
}

__global__ void k_pos_index(DevGraph g, uint4 *pidx, uint32_t *err, uint64_t p_lo, uint64_t p_hi) {
  for (uint64_t p = p_lo + blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < p_hi;
       p += uint64_t(gridDim.x) * blockDim.x) {
    bool bad = false;
    const uint64_t o0 = g.offsets[p], end = g.offsets[p + 1];
    BitReader r;
    r.seek(g.words, o0);
    const uint32_t nsi = r.segcnt(bad);
    const uint64_t ibase = r.pos();
    uint64_t last = r.pos();
    if (!bad && nsi && ibase + uint64_t(kSegBits) * (nsi - 1) < end) {
      // only the last interval segment is unpadded: decode it to find its end
      BitReader q;
      q.seek(g.words, ibase + uint64_t(kSegBits) * (nsi - 1));
      const uint32_t cnt = q.gamma(bad);
      for (uint32_t k = 0; k < cnt && !bad && q.pos() <= end; k++) {
        q.gamma(bad);
        q.gamma(bad);
      }
      last = q.pos();
    } else if (nsi) {
      bad = true;
    }
    uint32_t nsr = 0;
    uint64_t rbase = last;
    if (!bad && last <= end) {
      r.seek(g.words, last);
      nsr = r.segcnt(bad);
      rbase = r.pos();
    }
    if (bad || rbase > end || rbase - o0 > 0xFFFFFFFFull || (nsr && rbase + uint64_t(kSegBits) * (nsr - 1) >= end)) {
      set_error(err, kErrBadStream);
      pidx[p] = make_uint4(0u, 0u, 0u, 0u);
    } else {
      pidx[p] = make_uint4(uint32_t(ibase - o0), uint32_t(rbase - o0), nsi, nsr);
    }
  }
}

// Decode positions into a CSR scratch (parity hook).
__global__ void k_decode_positions(DecodeArgs a) {
  const DevGraph &g = a.g;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < a.n_pos;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t p = a.pos_list ? a.pos_list[i] : a.pos_begin + i;
    if (p >= g.n_c) continue;
    uint32_t *dst = a.out + a.arc_off[p];
    const uint64_t d = a.arc_off[p + 1] - a.arc_off[p];
    uint64_t k = 0;
    const int64_t r = walk_vertex(GWords{g.words}, g.offsets[p], g.offsets[p + 1], g.vertices[p], g.n,
                                  [&](uint32_t id) {
                                    if (k < d) dst[k] = id;
                                    k++;
                                  });
    if (r != int64_t(d)) {
      set_error(a.err, kErrBadStream);
      for (uint64_t q = (r > 0 ? uint64_t(r) : 0); q < d; q++) dst[q] = g.vertices[p];
    }
  }
}

__global__ void k_degree_count(DevGraph g, uint32_t *deg_out, uint32_t *itv_out, uint32_t *err, uint64_t p_lo,
                               uint64_t p_hi) {
  for (uint64_t p = p_lo + blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < p_hi;
       p += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t d = 0, itv = 0;
    if (g.vertices[p] >= g.n) {
      set_error(err, kErrBadStream);
    } else if (p < g.n_c) {
      int64_t iv = 0;
      const int64_t c = walk_vertex_buf(g.words, g.offsets[p], g.offsets[p + 1], g.vertices[p], g.n,
                                        [](uint32_t) {}, &iv);
      if (c < 0 || c > int64_t(0xFFFFFFFFll)) {
        set_error(err, kErrBadStream);
      } else {
        d = uint32_t(c);
        itv = uint32_t(iv);
      }
    } else {
      const uint32_t b = g.small_off[p - g.n_c], e = g.small_off[p - g.n_c + 1];
      if (e < b) {
        set_error(err, kErrBadStream);
      } else {
        d = e - b;
        for (uint32_t k = b; k < e; k++)
          if (g.small_nbr[k] >= g.n) {
            set_error(err, kErrBadStream);
            d = 0;
            break;
          }
      }
    }
    deg_out[p] = d;
    if (itv_out) itv_out[p] = itv;
  }
}

__global__ void k_init_labels(uint32_t *a, uint32_t *b, uint64_t n) {
  for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < n; v += uint64_t(gridDim.x) * blockDim.x) {
    a[v] = uint32_t(v);
    b[v] = uint32_t(v);
  }
}

#include "noalloc_kernels.cuh"  // kernels of lpa_iterate_noalloc

}  // namespace lpa_dev
