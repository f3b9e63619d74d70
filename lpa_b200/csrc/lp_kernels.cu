// Label-propagation kernels for sm_100a.
//
// One synchronous iteration reads lab_in and writes lab_out (double-buffered)
// for every vertex of degree > 0.  The update rule: the most frequent
// neighbour label, the smallest label on ties; vertices with degree >=
// cms_thr (cms_thr != 0) use a depth-4, width-1024 count-min sketch with
// seeded cm_hash rows (include/cms.cuh:96-132) and take the argmax of the
// sketch estimate over their neighbour labels, smallest label on ties.
//
// Work is organised in segments: contiguous ranges of positions (the
// vertices[] order of the compressed graph).  Each launch handles a list of
// segments; a block takes one segment at a time.
#include "lp_kernels.cuh"

namespace lpa_dev {

__device__ __forceinline__ uint32_t next_pow2(uint32_t x) {
  return x <= 1 ? 1u : (1u << (32 - __clz(x - 1)));
}

__device__ __forceinline__ void flush_changed(unsigned long long *counter, unsigned long long mine) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(kFull, mine, o);
  if ((threadIdx.x & 31) == 0 && mine) atomicAdd(counter, mine);
}

// ---------------------------------------------------------------------------
// V1 / V2: lane-per-vertex decode into a per-warp staging buffer, then count.
// ---------------------------------------------------------------------------
template <bool kPacked>
__device__ __forceinline__ void lane_batch(const IterArgs &a) {
  extern __shared__ uint32_t smem[];
  const int warp = threadIdx.x >> 5;
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t *stage = smem + warp * kStage;
  uint32_t *keys = smem + kLaneWarps * kStage + warp * (2 * kV1Slots);
  uint32_t *cnts = keys + kV1Slots;
  const DevGraph &g = a.g;
  const uint32_t *lab_in;
  uint32_t *lab_out;
  unsigned long long *counter;
  resolve_iter(a, lab_in, lab_out, counter);
  unsigned long long changed = 0;
  if (!kPacked) {  // tables start empty and are cleared after every vertex
    for (uint32_t i = lane; i < 2 * kV1Slots; i += 32) keys[i] = 0u;
    __syncwarp();
  }

  for (uint32_t li = blockIdx.x; li < a.n_list; li += gridDim.x) {
    const uint32_t s = a.seg_list[li];
    const Seg seg = a.segs[s];
    const long long t0 = clock64();
    const uint32_t nchunks = (seg.end - seg.begin + 31) / 32;
    for (uint32_t c = warp; c < nchunks; c += kLaneWarps) {
      const uint32_t p = seg.begin + c * 32 + lane;
      const bool valid = p < seg.end;
      const uint32_t node = valid ? g.vertices[p] : 0u;
      uint32_t d = valid ? g.deg[p] : 0u;
      const uint32_t old = valid ? __ldg(lab_in + node) : 0u;
      const bool cgr = valid && p < g.n_c;
      const uint32_t *items = nullptr;
      if (valid && !cgr) items = g.small_nbr + g.small_off[p - g.n_c];
      else if (cgr && a.from_scratch) items = a.scratch + a.arc_off[p];
      const bool need_stage = cgr && !a.from_scratch;
      if (kPacked ? d > kV2MaxDeg : d > kV1MaxDeg) {
        set_error(a.err, kErrCapacity);
        d = 0;
      }

      uint32_t done = ~__ballot_sync(kFull, valid);
      while (done != kFull) {
        const bool pending = !((done >> lane) & 1u);
        const uint32_t sd = (pending && need_stage) ? d : 0u;
        uint32_t incl = sd;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t t = __shfl_up_sync(kFull, incl, o);
          if (lane >= uint32_t(o)) incl += t;
        }
        const bool in_batch = pending && incl <= kStage;
        const uint32_t batch = __ballot_sync(kFull, in_batch);
        if (in_batch && need_stage) {
          const uint32_t base = incl - sd;
          uint32_t k = 0;
          const int64_t r = walk_vertex(GWords{g.words}, g.offsets[p], g.offsets[p + 1], node, g.n,
                                        [&](uint32_t id) {
                                          if (k < d) stage[base + k] = id;
                                          k++;
                                        });
          if (r != int64_t(d)) {
            set_error(a.err, kErrBadStream);
            for (uint32_t q = (r > 0 ? uint32_t(r) : 0u); q < d; q++) stage[base + q] = node;
          }
          items = stage + base;
        }
        __syncwarp();
        if (batch) {
          const uint32_t lo = __ffs(batch) - 1, hi = 32 - __clz(batch);
          if (kPacked) {
            // several vertices per round: G lanes per vertex
            const uint32_t dmax = __reduce_max_sync(kFull, ((batch >> lane) & 1u) ? d : 0u);
            const uint32_t G = next_pow2(dmax);
            const uint32_t per = 32 / G;
            const uint32_t gl = lane / G, k = lane % G;
            const uint32_t gm = (G == 32) ? kFull : (((1u << G) - 1u) << (gl * G));
            for (uint32_t v0 = lo; v0 < hi; v0 += per) {
              const uint32_t vi = v0 + gl;
              const bool vin = vi < hi;
              const uint32_t src = vin ? vi : lo;
              const uint32_t dv = __shfl_sync(kFull, d, src);
              const uint32_t *ip =
                  reinterpret_cast<const uint32_t *>(__shfl_sync(kFull, (unsigned long long)items, src));
              const uint32_t nodev = __shfl_sync(kFull, node, src);
              const uint32_t oldv = __shfl_sync(kFull, old, src);
              const bool ok = vin && k < dv;
              const uint32_t lab = ok ? __ldg(lab_in + ip[k]) : kFull;
              const uint32_t m = __match_any_sync(kFull, (uint64_t(gl) << 32) | lab);
              const uint32_t cnt = ok ? __popc(m) : 0u;
              const uint32_t maxc = __reduce_max_sync(gm, cnt);
              const uint32_t best = __reduce_min_sync(gm, (ok && cnt == maxc) ? lab : kFull);
              if (vin && k == 0) {
                const uint32_t nl = dv ? best : oldv;
                lab_out[nodev] = nl;
                changed += (nl != oldv);
              }
            }
          } else {
            // one vertex per round
            for (uint32_t j = lo; j < hi; j++) {
              const uint32_t dv = __shfl_sync(kFull, d, j);
              const uint32_t *ip =
                  reinterpret_cast<const uint32_t *>(__shfl_sync(kFull, (unsigned long long)items, j));
              const uint32_t nodev = __shfl_sync(kFull, node, j);
              const uint32_t oldv = __shfl_sync(kFull, old, j);
              uint32_t best;
              if (dv <= 32) {
                const bool ok = lane < dv;
                const uint32_t lab = ok ? __ldg(lab_in + ip[lane]) : kFull;
                const uint32_t m = __match_any_sync(kFull, lab);
                const uint32_t cnt = ok ? __popc(m) : 0u;
                const uint32_t maxc = __reduce_max_sync(kFull, cnt);
                best = __reduce_min_sync(kFull, (ok && cnt == maxc) ? lab : kFull);
              } else {
                const uint32_t cap = next_pow2(2 * dv);
                for (uint32_t k0 = 0; k0 < dv; k0 += 32) {
                  const uint32_t k = k0 + lane;
                  const bool ok = k < dv;
                  const uint32_t lab = ok ? __ldg(lab_in + ip[k]) : kFull;
                  const uint32_t m = __match_any_sync(kFull, lab);
                  if (ok && (__ffs(m) - 1) == int(lane)) table_add(keys, cnts, cap, lab, __popc(m));
                }
                __syncwarp();
                uint64_t bp = 0;
                for (uint32_t i = lane; i < cap; i += 32) {
                  const uint32_t kk = keys[i];
                  if (kk) {
                    const uint64_t cand = pack_best(cnts[i], kk - 1u);
                    bp = cand > bp ? cand : bp;
                    keys[i] = 0u;
                    cnts[i] = 0u;
                  }
                }
                best = best_label(warp_max_u64(bp));
                __syncwarp();
              }
              if (lane == 0) {
                const uint32_t nl = dv ? best : oldv;
                lab_out[nodev] = nl;
                changed += (nl != oldv);
              }
            }
          }
        }
        __syncwarp();
        done |= batch;
      }
    }
    if (a.seg_cycles) {
      __syncthreads();
      if (threadIdx.x == 0) a.seg_cycles[s] = clock64() - t0;
    }
  }
  flush_changed(counter, changed);
}

__global__ void __launch_bounds__(kLaneWarps * 32) k_lane_batch_packed(IterArgs a) { lane_batch<true>(a); }
__global__ void __launch_bounds__(kLaneWarps * 32) k_lane_batch_warp(IterArgs a) { lane_batch<false>(a); }

// ---------------------------------------------------------------------------
// V3: block per vertex.  Threads decode 256-bit segments in parallel; each
// step every thread contributes at most one item (one residual, or a share of
// the block-wide flattening of the step's intervals).
// ---------------------------------------------------------------------------
struct BlockShared {
  uint32_t left[kBlockThreads];
  uint32_t pref[kBlockThreads + 1];
  uint32_t wsum[kBlockThreads / 32];
  uint64_t red[kBlockThreads / 32];
  uint64_t res_start;
  uint64_t last_end;
  uint32_t bad;
  uint32_t items;
};

// Block-wide exclusive scan of v into sh.pref (pref[kBlockThreads] = total).
__device__ __forceinline__ uint32_t block_excl_scan(BlockShared &sh, uint32_t v) {
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t t = __shfl_up_sync(kFull, incl, o);
    if (lane >= uint32_t(o)) incl += t;
  }
  if (lane == 31) sh.wsum[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < kBlockThreads / 32 ? sh.wsum[lane] : 0u;
    uint32_t wi = w;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t t = __shfl_up_sync(kFull, wi, o);
      if (lane >= uint32_t(o)) wi += t;
    }
    if (lane < kBlockThreads / 32) sh.wsum[lane] = wi - w;
    if (lane == kBlockThreads / 32 - 1) sh.pref[kBlockThreads] = wi;
  }
  __syncthreads();
  const uint32_t ex = incl - v + sh.wsum[warp];
  sh.pref[threadIdx.x] = ex;
  __syncthreads();
  return sh.pref[kBlockThreads];
}

// Calls consume(ok, id) block-synchronously for every neighbour of position p.
template <class Consume>
__device__ __forceinline__ void block_for_each(const IterArgs &a, BlockShared &sh, uint32_t p, uint32_t node,
                                               uint32_t d, Consume consume) {
  const DevGraph &g = a.g;
  const uint32_t t = threadIdx.x;
  uint32_t my_items = 0;
  if (p >= g.n_c || a.from_scratch) {
    const uint32_t *ip = (p >= g.n_c) ? g.small_nbr + g.small_off[p - g.n_c] : a.scratch + a.arc_off[p];
    for (uint32_t k0 = 0; k0 < d; k0 += kBlockThreads) {
      const uint32_t k = k0 + t;
      const bool ok = k < d;
      consume(ok, ok ? ip[k] : 0u);
    }
    return;
  }
  const GWords W{g.words};
  const uint64_t end = g.offsets[p + 1];
  bool bad = false;
  uint64_t q = g.offsets[p];
  uint32_t nseg = dec_segcnt(W, q, bad);
  const uint64_t ibase = q;
  if (q > end || nseg > (end - q) / kSegBits + 1) {  // more segments than bits: malformed
    bad = true;
    nseg = 0;
  }
  if (t == 0) {
    sh.res_start = q;
    sh.bad = 0;
    sh.items = 0;
  }
  __syncthreads();
  // interval section
  for (uint32_t j0 = 0; j0 < nseg; j0 += kBlockThreads) {
    const uint32_t j = j0 + t;
    bool has = j < nseg;
    uint64_t sq = ibase + uint64_t(kSegBits) * j;
    uint32_t cnt = 0, c = 0, left = 0;
    if (has) {
      if (sq >= end) {
        bad = true;
        has = false;
      } else {
        cnt = dec_gamma(W, sq, bad);
      }
    }
    while (__syncthreads_or(has && c < cnt)) {
      uint32_t len = 0;
      if (has && c < cnt) {
        const uint32_t l = dec_gamma(W, sq, bad);
        left = (c == 0) ? zigzag_first(node, l) : left + l + 1u;
        len = dec_gamma(W, sq, bad) + kMinItv;
        c++;
        if (bad || sq > end || uint64_t(left) + len > g.n) {
          bad = true;
          len = 0;
          cnt = c;
        }
      }
      sh.left[t] = left;
      const uint32_t total = block_excl_scan(sh, len);
      if (has && len) left += len;
      for (uint32_t i0 = 0; i0 < total; i0 += kBlockThreads) {
        const uint32_t i = i0 + t;
        const bool ok = i < total;
        uint32_t id = 0;
        if (ok) {
          uint32_t lo = 0, hi = kBlockThreads - 1;
          while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (sh.pref[mid] <= i) lo = mid;
            else hi = mid - 1;
          }
          id = sh.left[lo] + (i - sh.pref[lo]);
          my_items++;
        }
        consume(ok, id);
      }
      __syncthreads();
    }
    if (has && j == nseg - 1) sh.res_start = sq;
  }
  __syncthreads();
  // residual section
  q = sh.res_start;
  uint32_t nres = dec_segcnt(W, q, bad);
  const uint64_t rbase = q;
  if (q > end || nres > (end - q) / kSegBits + 1) {
    bad = true;
    nres = 0;
  }
  if (t == 0) sh.last_end = q;
  __syncthreads();
  for (uint32_t j0 = 0; j0 < nres; j0 += kBlockThreads) {
    const uint32_t j = j0 + t;
    bool has = j < nres;
    uint64_t sq = rbase + uint64_t(kSegBits) * j;
    uint32_t cnt = 0, c = 0, v = 0;
    if (has) {
      if (sq >= end) {
        bad = true;
        has = false;
      } else {
        cnt = dec_gamma(W, sq, bad);
      }
    }
    while (__syncthreads_or(has && c < cnt)) {
      bool ok = has && c < cnt;
      if (ok) {
        const uint32_t x = dec_zeta3(W, sq, bad);
        v = (c == 0) ? zigzag_first(node, x) : v + x + 1u;
        c++;
        if (bad || sq > end || uint64_t(v) >= g.n) {
          bad = true;
          ok = false;
          cnt = c;
        } else {
          my_items++;
        }
      }
      consume(ok, v);
    }
    if (has && j == nres - 1) sh.last_end = sq;
  }
  if (my_items) atomicAdd(&sh.items, my_items);
  if (bad) sh.bad = 1;
  __syncthreads();
  if (t == 0 && (sh.bad || sh.last_end != end || sh.items != d)) set_error(a.err, kErrBadStream);
  __syncthreads();
}

__global__ void __launch_bounds__(kBlockThreads) k_block(IterArgs a) {
  extern __shared__ uint32_t smem[];
  __shared__ BlockShared sh;
  uint32_t *skeys = smem, *scnts = smem + kBlockSlots;
  uint32_t *cms = smem;  // depth x width counters share the table memory
  const DevGraph &g = a.g;
  const uint32_t t = threadIdx.x, lane = t & 31u, warp = t >> 5;
  const uint32_t *lab_in;
  uint32_t *lab_out;
  unsigned long long *counter;
  resolve_iter(a, lab_in, lab_out, counter);
  unsigned long long changed = 0;
  for (uint32_t i = t; i < 2 * kBlockSlots; i += kBlockThreads) smem[i] = 0u;  // tables start empty
  __syncthreads();

  for (uint32_t li = blockIdx.x; li < a.n_list; li += gridDim.x) {
    const uint32_t s = a.seg_list[li];
    const Seg seg = a.segs[s];
    const long long t0 = clock64();
    for (uint32_t p = seg.begin; p < seg.end; p++) {
      const uint32_t node = g.vertices[p];
      const uint32_t d = g.deg[p];
      const uint32_t old = __ldg(lab_in + node);
      if (d == 0) continue;
      const bool use_cms = a.cms_thr != 0 && d >= a.cms_thr;
      uint64_t bp = 0;
      if (use_cms) {
        block_for_each(a, sh, p, node, d, [&](bool ok, uint32_t id) {
          const uint32_t lab = ok ? __ldg(lab_in + id) : kFull;
          const uint32_t m = __match_any_sync(kFull, lab);
          if (ok && (__ffs(m) - 1) == int(lane)) {
            const uint32_t c = __popc(m);
#pragma unroll
            for (int r = 0; r < kCmsDepth; r++)
              atomicAdd(&cms[r * kCmsWidth + (cm_hash(r, lab ^ a.seeds[r]) & (kCmsWidth - 1))], c);
          }
        });
        __syncthreads();
        block_for_each(a, sh, p, node, d, [&](bool ok, uint32_t id) {
          if (ok) {
            const uint32_t lab = __ldg(lab_in + id);
            uint32_t est = kFull;
#pragma unroll
            for (int r = 0; r < kCmsDepth; r++) {
              const uint32_t cv = cms[r * kCmsWidth + (cm_hash(r, lab ^ a.seeds[r]) & (kCmsWidth - 1))];
              est = cv < est ? cv : est;
            }
            const uint64_t cand = pack_best(est, lab);
            bp = cand > bp ? cand : bp;
          }
        });
        __syncthreads();
        for (uint32_t i = t; i < kCmsDepth * kCmsWidth; i += kBlockThreads) cms[i] = 0u;
      } else {
        uint32_t *keys, *cnts;
        const uint32_t cap = next_pow2(2 * d);
        if (d <= kBlockMaxSmemDeg) {
          keys = skeys;
          cnts = scnts;
        } else {
          if (a.gtab_slots == 0 || cap > a.gtab_slots) {
            set_error(a.err, kErrCapacity);
            continue;
          }
          keys = a.gtab + uint64_t(blockIdx.x) * 2 * a.gtab_slots;
          cnts = keys + a.gtab_slots;
        }
        block_for_each(a, sh, p, node, d, [&](bool ok, uint32_t id) {
          const uint32_t lab = ok ? __ldg(lab_in + id) : kFull;
          const uint32_t m = __match_any_sync(kFull, lab);
          if (ok && (__ffs(m) - 1) == int(lane)) table_add(keys, cnts, cap, lab, __popc(m));
        });
        __syncthreads();
        for (uint32_t i = t; i < cap; i += kBlockThreads) {
          const uint32_t kk = keys[i];
          if (kk) {
            const uint64_t cand = pack_best(cnts[i], kk - 1u);
            bp = cand > bp ? cand : bp;
            keys[i] = 0u;
            cnts[i] = 0u;
          }
        }
      }
      bp = warp_max_u64(bp);
      if (lane == 0) sh.red[warp] = bp;
      __syncthreads();
      if (t == 0) {
        uint64_t b = 0;
        for (int w = 0; w < kBlockThreads / 32; w++) b = sh.red[w] > b ? sh.red[w] : b;
        const uint32_t nl = b ? best_label(b) : old;
        lab_out[node] = nl;
        changed += (nl != old);
      }
      __syncthreads();
    }
    if (a.seg_cycles && t == 0) a.seg_cycles[s] = clock64() - t0;
  }
  flush_changed(counter, changed);
}

// ---------------------------------------------------------------------------
// Decode positions into a CSR scratch (two-pass variant, parity hook).
// ---------------------------------------------------------------------------
__global__ void k_decode_positions(DecodeArgs a) {
  const DevGraph &g = a.g;
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < a.n_pos;
       i += uint64_t(gridDim.x) * blockDim.x) {
    const uint64_t p = a.pos_list ? a.pos_list[i] : i;
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

// Two-pass variant, pass 1: block per segment, thread per position.
__global__ void k_decode_segments(IterArgs a) {
  const DevGraph &g = a.g;
  for (uint32_t li = blockIdx.x; li < a.n_list; li += gridDim.x) {
    const Seg seg = a.segs[a.seg_list[li]];
    for (uint32_t p = seg.begin + threadIdx.x; p < seg.end; p += blockDim.x) {
      if (p >= g.n_c) continue;
      uint32_t *dst = const_cast<uint32_t *>(a.scratch) + a.arc_off[p];
      const uint32_t d = g.deg[p];
      uint32_t k = 0;
      const int64_t r = walk_vertex(GWords{g.words}, g.offsets[p], g.offsets[p + 1], g.vertices[p], g.n,
                                    [&](uint32_t id) {
                                      if (k < d) dst[k] = id;
                                      k++;
                                    });
      if (r != int64_t(d)) {
        set_error(a.err, kErrBadStream);
        for (uint32_t q = (r > 0 ? uint32_t(r) : 0u); q < d; q++) dst[q] = g.vertices[p];
      }
    }
  }
}

__global__ void k_degree_count(DevGraph g, uint32_t *deg_out, uint32_t *err) {
  for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < g.n;
       p += uint64_t(gridDim.x) * blockDim.x) {
    uint32_t d = 0;
    if (g.vertices[p] >= g.n) {
      set_error(err, kErrBadStream);
    } else if (p < g.n_c) {
      const int64_t c = walk_vertex(GWords{g.words}, g.offsets[p], g.offsets[p + 1], g.vertices[p], g.n,
                                    [](uint32_t) {});
      if (c < 0 || c > int64_t(0xFFFFFFFFll)) set_error(err, kErrBadStream);
      else d = uint32_t(c);
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
  }
}

__global__ void k_init_labels(uint32_t *a, uint32_t *b, uint64_t n) {
  for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < n; v += uint64_t(gridDim.x) * blockDim.x) {
    a[v] = uint32_t(v);
    b[v] = uint32_t(v);
  }
}

}  // namespace lpa_dev
