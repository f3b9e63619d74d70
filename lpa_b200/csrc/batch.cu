// Batched graphs: many independent graphs propagated by one persistent launch
// (k_batch) fed by a device ring queue, each graph with its own convergence
// test.  Graph arrays are packed into one device allocation per kind; every
// graph keeps its own labels, segments and fixed degree-bucket plan.
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
  if (b->stream) cudaStreamSynchronize(b->stream);
  for (void *p : b->allocs) cudaFree(p);
  if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
  cudaGetLastError();
  delete b;
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
                       b->stream>>>(bg.g, d_deg + ov, nullptr, b->d_err);
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
        a.spin_limit = 1ull << 25;  // ~7 s of 200 ns sleeps with nothing to do
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
  if (!b || graph >= b->graphs.size() || !host_out || n != b->n[graph]) return LPA_ERR_INVALID_ARG;
  const BatchGraph &bg = b->graphs[graph];
  const uint32_t *src = (b->iters[graph] & 1u) ? bg.labs1 : bg.labs0;
  if (cudaSetDevice(b->device) != cudaSuccess ||
      cudaMemcpy(host_out, src, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess) {
    cudaGetLastError();
    return LPA_ERR_CUDA;
  }
  return LPA_OK;
}

lpa_status lpa_batch_destroy(lpa_batch *b) {
  if (!b) return LPA_ERR_INVALID_ARG;
  free_batch(b);
  return LPA_OK;
}

}  // extern "C"
