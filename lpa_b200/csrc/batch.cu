// Batched graphs, each with its own convergence test, in one of two modes.
//
// Lockstep (the default): the batch is concatenated into one graph whose
// vertex ids are shifted per graph, and that graph runs through the ordinary
// handle (every variant, the learned plan, the autotuner and the CUDA-graph
// loop) while a two-launch tracker after every iteration records which graphs
// changed.  Labels are compared, never added, so the shift changes no exact
// count; the sketch hashes labels relative to their graph's base
// (IterArgs::gbase), so its counts are those of each graph alone.  A graph
// that did not change has reached a fixed point: later iterations rewrite
// the same labels, so its result and iteration count are the ones it has run
// alone, and the loop ends when every graph has stopped.
//
// Queue: one persistent launch (k_batch) fed by a device ring queue; every
// graph keeps its own labels, segments and fixed degree-bucket plan and
// leaves the queue as soon as it converges.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "lp_kernels.cuh"
#include "runtime.h"

using namespace lpa_dev;

struct lpa_batch {
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  lpa_opts opts{};
  int num_sms = 148, occ = 1;
  std::vector<uint64_t> n, n_c;
  std::vector<void *> allocs;
  BatchGraph *d_graphs = nullptr;
  std::vector<BatchGraph> graphs;
  unsigned long long *d_queue = nullptr, *d_head = nullptr, *d_tail = nullptr, *d_changed = nullptr;
  uint32_t *d_active = nullptr, *d_done = nullptr, *d_iters = nullptr, *d_err = nullptr;
  uint32_t *d_gtab = nullptr, gtab_slots = 0;
  uint32_t cap = 0;
  std::vector<uint32_t> iters;
  std::vector<unsigned long long> initial_queue;
  uint32_t seeds[kCmsDepth];
  std::string last_error;
  // lockstep mode: the concatenated graph and each graph's first vertex id
  lpa_handle *h = nullptr;
  std::vector<uint32_t> gbase;
};

namespace {

template <class T>
T *balloc(lpa_batch *b, uint64_t count) {
  void *p = nullptr;
  if (cudaMalloc(&p, std::max<uint64_t>(1, count) * sizeof(T)) != cudaSuccess) {
    cudaGetLastError();
    throw LPA_ERR_OOM;
  }
  b->allocs.push_back(p);
  return static_cast<T *>(p);
}

void bcheck(cudaError_t e) {
  if (e != cudaSuccess) throw(e == cudaErrorMemoryAllocation ? LPA_ERR_OOM : LPA_ERR_CUDA);
}

void free_batch(lpa_batch *b) {
  if (!b) return;
  if (b->h) {
    lpa_destroy(b->h);
    delete b;
    return;
  }
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (void *p : b->allocs) cudaFree(p);
  if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
  cudaGetLastError();
  delete b;
}

// ------------------------------------------------------------ lockstep ----
// The batch as one graph (lpa_hg_concat) and where each graph lies in it.
struct Union {
  lpa_host_graph *hg = nullptr;
  lpa_graph_desc desc{};
  std::vector<uint32_t> gbase;         // G + 1 vertex-id starts
  std::vector<uint64_t> cbase, sbase;  // G + 1 compressed / small position starts
  ~Union() {
    if (hg) lpa_hg_free(hg);
  }
};

// LPA_ERR_CAPACITY when the concatenation's ids leave 32 bits.
lpa_status build_union(const lpa_graph_desc *graphs, size_t G, Union &u) {
  lpa_status st = lpa_hg_concat(graphs, G, &u.hg);
  if (st != LPA_OK) return st;
  st = lpa_hg_desc(u.hg, &u.desc);
  if (st != LPA_OK) return st;
  u.gbase.assign(G + 1, 0);
  u.cbase.assign(G + 1, 0);
  u.sbase.assign(G + 1, 0);
  for (size_t gi = 0; gi < G; gi++) {
    u.gbase[gi + 1] = u.gbase[gi] + uint32_t(graphs[gi].num_vertices);
    u.cbase[gi + 1] = u.cbase[gi] + graphs[gi].num_compressed;
    u.sbase[gi + 1] = u.sbase[gi] + graphs[gi].num_vertices - graphs[gi].num_compressed;
  }
  return LPA_OK;
}

__device__ __forceinline__ uint32_t owner(const uint64_t *base, uint32_t G, uint64_t x) {
  uint32_t lo = 0, hi = G;  // base[lo] <= x < base[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (base[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Every position's vertex and neighbours lie in its own graph's id range
// (the handle's own pass checked them against the whole batch only).
__global__ void k_union_check(DevGraph g, const uint32_t *gbase, const uint64_t *cbase, const uint64_t *sbase,
                              uint32_t G, uint32_t *err) {
  for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < g.n; p += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t k = p < g.n_c ? owner(cbase, G, p) : owner(sbase, G, p - g.n_c);
    const uint32_t lo = gbase[k], hi = gbase[k + 1];
    const uint32_t node = g.vertices[p];
    bool bad = node < lo || node >= hi;
    if (!bad && p < g.n_c) {
      int64_t iv = 0;
      walk_vertex_buf(g.words, g.offsets[p], g.offsets[p + 1], node, g.n,
                      [&](uint32_t v) { bad |= v < lo || v >= hi; }, &iv);
    } else if (!bad) {
      for (uint32_t e = g.small_off[p - g.n_c]; e < g.small_off[p - g.n_c + 1]; e++) {
        const uint32_t v = g.small_nbr[e];
        bad |= v < lo || v >= hi;
      }
    }
    if (bad) atomicExch(err, 1u);
  }
}

// Marks every graph with a vertex whose two label buffers differ: after an
// iteration these are its changed vertices (vertices without neighbours hold
// the same label in both).
__global__ void k_track_changed(const uint32_t *__restrict__ l0, const uint32_t *__restrict__ l1, uint64_t n,
                                const uint32_t *__restrict__ gbase, uint32_t G, uint32_t *flags) {
  uint32_t glo = 1, ghi = 0;  // the last owner found: ids [glo, ghi)
  const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
  for (uint64_t v0 = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v0 < n; v0 += 4 * stride) {
    uint32_t a[4], b[4];
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint64_t v = v0 + u * stride;
      a[u] = v < n ? __ldcs(l0 + v) : 0u;
      b[u] = v < n ? __ldcs(l1 + v) : 0u;
    }
#pragma unroll
    for (int u = 0; u < 4; u++) {
      const uint32_t v = uint32_t(v0 + u * stride);
      if (a[u] == b[u] || (v >= glo && v < ghi)) continue;  // unchanged, or its graph is marked
      uint32_t lo = 0, hi = G;
      while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(gbase + mid) <= v) lo = mid;
        else hi = mid;
      }
      glo = __ldg(gbase + lo);
      ghi = __ldg(gbase + lo + 1);
      flags[lo] = 1u;
    }
  }
}

// Ends the iteration for the tracker: a running graph whose flag is clear (or
// that reached max_iter) records the iterations done; flags are cleared.
__global__ void k_track_step(uint32_t *track, uint32_t G) {
  __shared__ uint32_t s_it;
  if (threadIdx.x == 0) s_it = track[0] + 1u;
  __syncthreads();
  const uint32_t it = s_it, max_iter = track[1], early = track[2];
  uint32_t *flags = track + 4, *done = track + 4 + G;
  for (uint32_t k = threadIdx.x; k < G; k += blockDim.x) {
    if (done[k] == 0u && ((early && flags[k] == 0u) || it >= max_iter)) done[k] = it;
    flags[k] = 0u;
  }
  if (threadIdx.x == 0) track[0] = it;
}

}  // namespace

void lpa_rt_enqueue_track(lpa_handle *h) {
  const int blocks = int(std::max<uint64_t>(1, std::min<uint64_t>((h->n + 1023) / 1024, uint64_t(h->num_sms) * 8)));
  k_track_changed<<<blocks, 256, 0, h->stream>>>(h->d_lab[0], h->d_lab[1], h->n, h->d_gbase, h->n_graphs,
                                                 h->d_gtrack + 4);
  k_track_step<<<1, 1024, 0, h->stream>>>(h->d_gtrack, h->n_graphs);
}

namespace {

// Lockstep create: the union handle plus the tracker's memory.
lpa_status create_lockstep(lpa_batch *b, const lpa_graph_desc *graphs, size_t G, const Union &u) {
  lpa_handle *h = nullptr;
  lpa_status st = lpa_create(&u.desc, &b->opts, &h);
  if (st != LPA_OK) return st;
  b->h = h;
  b->device = h->device;
  b->stream = h->stream;
  b->own_stream = false;
  auto dev = [&](size_t bytes) -> void * {
    void *p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(bytes, 4)) != cudaSuccess) {
      cudaGetLastError();
      throw LPA_ERR_OOM;
    }
    h->allocations.push_back(p);
    return p;
  };
  try {
    h->d_gbase = static_cast<uint32_t *>(dev((G + 1) * 4));
    uint64_t *d_cbase = static_cast<uint64_t *>(dev((G + 1) * 8));
    uint64_t *d_sbase = static_cast<uint64_t *>(dev((G + 1) * 8));
    h->d_gtrack = static_cast<uint32_t *>(dev((4 + 2 * G) * 4));
    bcheck(cudaMemcpyAsync(h->d_gbase, u.gbase.data(), (G + 1) * 4, cudaMemcpyHostToDevice, h->stream));
    bcheck(cudaMemcpyAsync(d_cbase, u.cbase.data(), (G + 1) * 8, cudaMemcpyHostToDevice, h->stream));
    bcheck(cudaMemcpyAsync(d_sbase, u.sbase.data(), (G + 1) * 8, cudaMemcpyHostToDevice, h->stream));
    bcheck(cudaMemsetAsync(h->d_gtrack, 0, (4 + 2 * G) * 4, h->stream));
    bcheck(cudaMemsetAsync(h->d_err, 0, 4, h->stream));
    DevGraph g;
    g.words = h->d_words;
    g.offsets = h->d_offsets;
    g.vertices = h->d_vertices;
    g.deg = h->d_deg;
    g.small_off = h->d_small_off;
    g.small_nbr = h->d_small_nbr;
    g.n = h->n;
    g.n_c = h->n_c;
    const int blocks = int(std::max<uint64_t>(1, std::min<uint64_t>((h->n + 127) / 128, uint64_t(h->num_sms) * 16)));
    k_union_check<<<blocks, 128, 0, h->stream>>>(g, h->d_gbase, d_cbase, d_sbase, uint32_t(G), h->d_err);
    bcheck(cudaGetLastError());
    uint32_t err = 0;
    bcheck(cudaMemcpyAsync(&err, h->d_err, 4, cudaMemcpyDeviceToHost, h->stream));
    bcheck(cudaStreamSynchronize(h->stream));
    if (err) throw LPA_ERR_BAD_STREAM;
  } catch (lpa_status e) {
    return e;
  }
  h->n_graphs = uint32_t(G);
  b->gbase = u.gbase;
  for (size_t gi = 0; gi < G; gi++) {
    b->n.push_back(graphs[gi].num_vertices);
    b->n_c.push_back(graphs[gi].num_compressed);
  }
  b->iters.assign(G, 0);
  return LPA_OK;
}

lpa_status run_lockstep(lpa_batch *b, int max_iter, int early_exit, uint32_t *iters_per_graph) {
  lpa_handle *h = b->h;
  const size_t G = b->gbase.size() - 1;
  lpa_status st = lpa_init_labels(h);
  if (st != LPA_OK) return st;
  try {
    const uint32_t ctl[4] = {0u, uint32_t(max_iter), early_exit ? 1u : 0u, 0u};
    bcheck(cudaMemsetAsync(h->d_gtrack, 0, (4 + 2 * G) * 4, h->stream));
    bcheck(cudaMemcpyAsync(h->d_gtrack, ctl, sizeof(ctl), cudaMemcpyHostToDevice, h->stream));
  } catch (lpa_status e) {
    return e;
  }
  int done = 0;
  st = lpa_run(h, max_iter, early_exit, &done);
  if (st != LPA_OK) return st;
  std::vector<uint32_t> it(G, 0);
  if (cudaMemcpyAsync(it.data(), h->d_gtrack + 4 + G, G * 4, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess) {
    cudaGetLastError();
    return LPA_ERR_CUDA;
  }
  // graphs still marked running ran every iteration of the loop
  for (size_t gi = 0; gi < G; gi++) b->iters[gi] = it[gi] ? it[gi] : uint32_t(done);
  if (iters_per_graph) std::memcpy(iters_per_graph, b->iters.data(), G * 4);
  return LPA_OK;
}

}  // namespace

extern "C" {

lpa_status lpa_batch_create(const lpa_graph_desc *graphs, size_t num_graphs, const lpa_opts *o, lpa_batch **out) {
  if (!graphs || !out || num_graphs == 0 || num_graphs >= (1u << 20)) return LPA_ERR_INVALID_ARG;
  *out = nullptr;
  for (size_t gi = 0; gi < num_graphs; gi++) {
    const lpa_graph_desc &g = graphs[gi];
    if (g.num_vertices == 0 || g.num_vertices > 0xFFFFFFFEull || g.num_compressed > g.num_vertices || !g.vertices)
      return LPA_ERR_INVALID_ARG;
    if (g.num_compressed && (!g.words || !g.offsets || g.offsets[0] != 0)) return LPA_ERR_INVALID_ARG;
    for (uint64_t i = 0; i < g.num_compressed; i++)
      if (g.offsets[i + 1] < g.offsets[i]) return LPA_ERR_BAD_STREAM;
    if (g.num_compressed && (g.offsets[g.num_compressed] + 31) / 32 > g.num_words) return LPA_ERR_BAD_STREAM;
    if (g.num_vertices > g.num_compressed &&
        (!g.small_offset || g.small_offset[0] != 0 || g.small_offset[g.num_vertices - g.num_compressed] != g.num_small_arcs))
      return LPA_ERR_INVALID_ARG;
  }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return LPA_ERR_NO_DEVICE;
  }
  lpa_batch *b = new lpa_batch();
  if (o) b->opts = *o;
  else lpa_opts_default(&b->opts);
  if (b->opts.stream_budget != 0) {  // out-of-core streaming serves single graphs only
    delete b;
    return LPA_ERR_INVALID_ARG;
  }
  if (b->opts.batch_mode == LPA_BATCH_LOCKSTEP) {
    Union u;
    lpa_status st = build_union(graphs, num_graphs, u);
    if (st == LPA_OK) st = create_lockstep(b, graphs, num_graphs, u);
    if (st != LPA_ERR_CAPACITY) {  // past 32-bit ids the queue keeps every graph's own ids
      if (st != LPA_OK) {
        free_batch(b);
        return st;
      }
      *out = b;
      return LPA_OK;
    }
  } else if (b->opts.batch_mode != LPA_BATCH_QUEUE) {
    delete b;
    return LPA_ERR_INVALID_ARG;
  }
  try {
    if (b->opts.device < 0 || b->opts.device >= count) throw LPA_ERR_INVALID_ARG;
    b->device = b->opts.device;
    bcheck(cudaSetDevice(b->device));
    if (b->opts.stream) {
      b->stream = static_cast<cudaStream_t>(b->opts.stream);
      b->own_stream = false;
    } else {
      bcheck(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    }
    bcheck(cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device));
    bcheck(cudaFuncSetAttribute(k_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmemBytes)));
    bcheck(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b->occ, k_batch, kThreads, kSmemBytes));
    b->occ = std::max(1, b->occ);
    const uint32_t lo = uint32_t(b->opts.cms_seed), hi = uint32_t(b->opts.cms_seed >> 32);
    for (int r = 0; r < kCmsDepth; r++) b->seeds[r] = (lo ^ (0x9E3779B9u * uint32_t(r + 1))) + hi * 0x85EBCA6Bu;
    // packed sizes
    uint64_t words = 0, offs = 0, verts = 0, soff = 0, snbr = 0;
    for (size_t gi = 0; gi < num_graphs; gi++) {
      const lpa_graph_desc &g = graphs[gi];
      words += g.num_words + 4;
      offs += g.num_compressed + 1;
      verts += g.num_vertices;
      soff += g.num_vertices - g.num_compressed + 1;
      snbr += g.num_small_arcs;
    }
    uint32_t *d_words = balloc<uint32_t>(b, words);
    bcheck(cudaMemsetAsync(d_words, 0, words * 4, b->stream));
    uint64_t *d_offs = balloc<uint64_t>(b, offs);
    uint32_t *d_verts = balloc<uint32_t>(b, verts);
    uint32_t *d_deg = balloc<uint32_t>(b, verts);
    uint32_t *d_soff = balloc<uint32_t>(b, soff);
    bcheck(cudaMemsetAsync(d_soff, 0, soff * 4, b->stream));
    uint32_t *d_snbr = balloc<uint32_t>(b, snbr);
    uint32_t *d_labs = balloc<uint32_t>(b, 2 * verts);
    b->d_err = balloc<uint32_t>(b, 1);
    bcheck(cudaMemsetAsync(b->d_err, 0, 4, b->stream));
    b->graphs.resize(num_graphs);
    uint64_t ow = 0, oo = 0, ov = 0, os = 0, on = 0;
    for (size_t gi = 0; gi < num_graphs; gi++) {
      const lpa_graph_desc &g = graphs[gi];
      BatchGraph &bg = b->graphs[gi];
      bg.g.words = d_words + ow;
      bg.g.offsets = d_offs + oo;
      bg.g.vertices = d_verts + ov;
      bg.g.deg = d_deg + ov;
      bg.g.small_off = d_soff + os;
      bg.g.small_nbr = d_snbr + on;
      bg.g.n = g.num_vertices;
      bg.g.n_c = g.num_compressed;
      bg.labs0 = d_labs + 2 * ov;
      bg.labs1 = d_labs + 2 * ov + g.num_vertices;
      if (g.num_words) bcheck(cudaMemcpyAsync(d_words + ow, g.words, g.num_words * 4, cudaMemcpyHostToDevice, b->stream));
      if (g.num_compressed)
        bcheck(cudaMemcpyAsync(d_offs + oo, g.offsets, (g.num_compressed + 1) * 8, cudaMemcpyHostToDevice, b->stream));
      bcheck(cudaMemcpyAsync(d_verts + ov, g.vertices, g.num_vertices * 4, cudaMemcpyHostToDevice, b->stream));
      if (g.num_vertices > g.num_compressed)
        bcheck(cudaMemcpyAsync(d_soff + os, g.small_offset, (g.num_vertices - g.num_compressed + 1) * 4,
                               cudaMemcpyHostToDevice, b->stream));
      if (g.num_small_arcs)
        bcheck(cudaMemcpyAsync(d_snbr + on, g.small_graph, g.num_small_arcs * 4, cudaMemcpyHostToDevice, b->stream));
      k_degree_count<<<std::max<uint64_t>(1, std::min<uint64_t>((g.num_vertices + 127) / 128, 4096)), 128, 0,
                       b->stream>>>(bg.g, d_deg + ov, nullptr, b->d_err, 0, g.num_vertices);
      ow += g.num_words + 4;
      oo += g.num_compressed + 1;
      ov += g.num_vertices;
      os += g.num_vertices - g.num_compressed + 1;
      on += g.num_small_arcs;
      b->n.push_back(g.num_vertices);
      b->n_c.push_back(g.num_compressed);
    }
    bcheck(cudaGetLastError());
    uint32_t err = 0;
    bcheck(cudaMemcpyAsync(&err, b->d_err, 4, cudaMemcpyDeviceToHost, b->stream));
    bcheck(cudaStreamSynchronize(b->stream));
    if (err) throw LPA_ERR_BAD_STREAM;
    // plans
    std::vector<uint32_t> deg(verts);
    bcheck(cudaMemcpy(deg.data(), d_deg, verts * 4, cudaMemcpyDeviceToHost));
    std::vector<Seg> all_segs;
    std::vector<uint8_t> all_var;
    std::vector<uint64_t> seg_off(num_graphs + 1, 0);
    uint64_t big = 0;
    ov = 0;
    for (size_t gi = 0; gi < num_graphs; gi++) {
      auto segs = lpa_rt::make_segments(deg.data() + ov, b->n[gi], b->n_c[gi], b->opts.cms_threshold);
      seg_off[gi + 1] = seg_off[gi] + segs.size();
      for (auto &sg : segs) {
        all_segs.push_back(Seg{sg.begin, sg.end});
        int v = lpa_rt::fixed_variant(sg);
        if (b->opts.dispatch == LPA_DISPATCH_FORCE && b->opts.force_variant != LPA_VARIANT_TWO_PASS &&
            lpa_rt::variant_capable(b->opts.force_variant, sg, b->opts.cms_threshold))
          v = b->opts.force_variant;
        // tiny packed segments run one thread per position
        if (v == LPA_VARIANT_PACKED && sg.max_deg <= kPackedMaxDeg) v = kVarPackedLanes;
        all_var.push_back(uint8_t(v));
      }
      for (uint64_t p = 0; p < b->n[gi]; p++) {
        const uint32_t d = deg[ov + p];
        const bool cms = b->opts.cms_threshold != 0 && d >= b->opts.cms_threshold;
        if (!cms && d > kBlockMaxSmemDeg) big = std::max<uint64_t>(big, d);
      }
      ov += b->n[gi];
    }
    Seg *d_segs = balloc<Seg>(b, all_segs.size());
    uint8_t *d_var = balloc<uint8_t>(b, all_var.size());
    bcheck(cudaMemcpyAsync(d_segs, all_segs.data(), all_segs.size() * sizeof(Seg), cudaMemcpyHostToDevice, b->stream));
    bcheck(cudaMemcpyAsync(d_var, all_var.data(), all_var.size(), cudaMemcpyHostToDevice, b->stream));
    uint64_t total_items = 0;
    for (size_t gi = 0; gi < num_graphs; gi++) {
      b->graphs[gi].segs = d_segs + seg_off[gi];
      b->graphs[gi].seg_var = d_var + seg_off[gi];
      b->graphs[gi].nseg = uint32_t(seg_off[gi + 1] - seg_off[gi]);
      total_items += b->graphs[gi].nseg;
    }
    if (total_items + 64 > 0xFFFFFFFFull) throw LPA_ERR_INVALID_ARG;
    b->cap = uint32_t(total_items + 64);
    int grid = b->num_sms * b->occ;
    if (big) {
      b->gtab_slots = lpa_rt::next_pow2_host(2 * big);
      const uint64_t per_block = uint64_t(b->gtab_slots) * 8;
      grid = int(std::max<uint64_t>(1, std::min<uint64_t>(uint64_t(grid), (2ull << 30) / per_block)));
      b->d_gtab = balloc<uint32_t>(b, uint64_t(grid) * 2 * b->gtab_slots);
      bcheck(cudaMemsetAsync(b->d_gtab, 0, uint64_t(grid) * per_block, b->stream));
    }
    b->occ = std::max(1, grid / b->num_sms);
    b->d_graphs = balloc<BatchGraph>(b, num_graphs);
    bcheck(cudaMemcpyAsync(b->d_graphs, b->graphs.data(), num_graphs * sizeof(BatchGraph), cudaMemcpyHostToDevice,
                           b->stream));
    b->d_queue = balloc<unsigned long long>(b, b->cap);
    b->d_head = balloc<unsigned long long>(b, 2);
    b->d_tail = b->d_head + 1;
    b->d_active = balloc<uint32_t>(b, 1);
    b->d_done = balloc<uint32_t>(b, num_graphs);
    b->d_changed = balloc<unsigned long long>(b, num_graphs);
    b->d_iters = balloc<uint32_t>(b, num_graphs);
    b->initial_queue.reserve(total_items);
    for (size_t gi = 0; gi < num_graphs; gi++)
      for (uint32_t s = 0; s < b->graphs[gi].nseg; s++) b->initial_queue.push_back((uint64_t(gi) << 44) | s);
    b->iters.assign(num_graphs, 0);
    bcheck(cudaStreamSynchronize(b->stream));
  } catch (lpa_status st) {
    b->last_error = "lpa_batch_create failed";
    free_batch(b);
    return st;
  }
  *out = b;
  return LPA_OK;
}

lpa_status lpa_batch_run(lpa_batch *b, int max_iter, int early_exit, uint32_t *iters_per_graph) {
  if (!b || max_iter < 0 || max_iter >= 4096) return LPA_ERR_INVALID_ARG;
  if (b->h) return run_lockstep(b, max_iter, early_exit, iters_per_graph);
  const size_t G = b->graphs.size();
  try {
    bcheck(cudaSetDevice(b->device));
    k_batch_init<<<int(std::min<size_t>(G, 4096)), 256, 0, b->stream>>>(b->d_graphs, uint32_t(G));
    bcheck(cudaGetLastError());
    std::fill(b->iters.begin(), b->iters.end(), 0u);
    if (max_iter == 0) {
      bcheck(cudaStreamSynchronize(b->stream));
    } else {
      // graphs without a single edge finish in one iteration that changes nothing
      std::vector<unsigned long long> q;
      q.reserve(b->initial_queue.size());
      uint32_t active = 0;
      for (size_t gi = 0; gi < G; gi++) {
        if (b->graphs[gi].nseg == 0) b->iters[gi] = 1;
        else active++;
      }
      bcheck(cudaMemsetAsync(b->d_queue, 0xFF, size_t(b->cap) * 8, b->stream));
      bcheck(cudaMemcpyAsync(b->d_queue, b->initial_queue.data(), b->initial_queue.size() * 8, cudaMemcpyHostToDevice,
                             b->stream));
      const unsigned long long ht[2] = {0ull, (unsigned long long)b->initial_queue.size()};
      bcheck(cudaMemcpyAsync(b->d_head, ht, 16, cudaMemcpyHostToDevice, b->stream));
      bcheck(cudaMemcpyAsync(b->d_active, &active, 4, cudaMemcpyHostToDevice, b->stream));
      bcheck(cudaMemsetAsync(b->d_done, 0, G * 4, b->stream));
      bcheck(cudaMemsetAsync(b->d_changed, 0, G * 8, b->stream));
      bcheck(cudaMemsetAsync(b->d_iters, 0, G * 4, b->stream));
      bcheck(cudaMemsetAsync(b->d_err, 0, 4, b->stream));
      if (active) {
        BatchArgs a{};
        a.graphs = b->d_graphs;
        a.ngraphs = uint32_t(G);
        a.queue = b->d_queue;
        a.cap = b->cap;
        a.head = b->d_head;
        a.tail = b->d_tail;
        a.active = b->d_active;
        a.done_items = b->d_done;
        a.changed = b->d_changed;
        a.iters = b->d_iters;
        a.err = b->d_err;
        a.max_iter = uint32_t(max_iter);
        a.early_exit = early_exit ? 1 : 0;
        a.cms_thr = b->opts.cms_threshold;
        for (int r = 0; r < kCmsDepth; r++) a.seeds[r] = b->seeds[r];
        a.gtab = b->d_gtab;
        a.gtab_slots = b->gtab_slots;
        // ~7 s of 200 ns sleeps with nothing to do, unless the caller bounds it
        a.spin_limit = b->opts.queue_wait_limit ? b->opts.queue_wait_limit : (1ull << 25);
        k_batch<<<b->num_sms * b->occ, kThreads, kSmemBytes, b->stream>>>(a);
        bcheck(cudaGetLastError());
      }
      std::vector<uint32_t> it(G);
      bcheck(cudaMemcpyAsync(it.data(), b->d_iters, G * 4, cudaMemcpyDeviceToHost, b->stream));
      uint32_t err = 0;
      bcheck(cudaMemcpyAsync(&err, b->d_err, 4, cudaMemcpyDeviceToHost, b->stream));
      bcheck(cudaStreamSynchronize(b->stream));
      for (size_t gi = 0; gi < G; gi++)
        if (b->graphs[gi].nseg) b->iters[gi] = it[gi];
      if (err == kErrTimeout) throw LPA_ERR_TIMEOUT;
      if (err == kErrCapacity) throw LPA_ERR_CAPACITY;
      if (err) throw LPA_ERR_BAD_STREAM;
    }
    if (iters_per_graph) std::memcpy(iters_per_graph, b->iters.data(), G * 4);
  } catch (lpa_status st) {
    return st;
  }
  return LPA_OK;
}

lpa_status lpa_batch_get_labels(lpa_batch *b, size_t graph, uint32_t *host_out, size_t n) {
  if (!b || graph >= b->n.size() || !host_out || n != b->n[graph]) return LPA_ERR_INVALID_ARG;
  if (b->h) {
    lpa_handle *h = b->h;
    const uint32_t base = b->gbase[graph];
    if (cudaSetDevice(h->device) != cudaSuccess ||
        cudaMemcpyAsync(host_out, h->d_lab[h->cur] + base, n * 4, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess ||
        cudaStreamSynchronize(h->stream) != cudaSuccess) {
      cudaGetLastError();
      return LPA_ERR_CUDA;
    }
    for (size_t i = 0; i < n; i++) host_out[i] -= base;
    return LPA_OK;
  }
  const BatchGraph &bg = b->graphs[graph];
  const uint32_t *src = (b->iters[graph] & 1u) ? bg.labs1 : bg.labs0;
  if (cudaSetDevice(b->device) != cudaSuccess ||
      cudaMemcpy(host_out, src, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return LPA_ERR_CUDA;
  }
  return LPA_OK;
}

lpa_handle *lpa_batch_handle(lpa_batch *b) { return b ? b->h : nullptr; }

lpa_status lpa_batch_destroy(lpa_batch *b) {
  if (!b) return LPA_ERR_INVALID_ARG;
  free_batch(b);
  return LPA_OK;
}

}  // extern "C"
