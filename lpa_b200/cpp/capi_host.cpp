// C ABI of the host format layer (lpa_hg_*): generators, the fast
// bit-identical CGR encoder and the reference's file formats.
#include <algorithm>
#include <new>
#include <stdexcept>
#include <string>

#include "lpa/cgr_format.h"
#include "lpa/generators.h"
#include "lpa_capi.h"

struct lpa_host_graph {
  lpa::CsrGraph csr;
  bool has_csr = false;
  lpa::CgrGraph cgr;
  bool has_cgr = false;
};

namespace {

template <class Fn>
lpa_status guarded(Fn fn) {
  try {
    return fn();
  } catch (const std::bad_alloc &) {
    return LPA_ERR_OOM;
  } catch (const std::invalid_argument &) {
    return LPA_ERR_INVALID_ARG;
  } catch (const std::runtime_error &) {
    return LPA_ERR_IO;
  } catch (...) {
    return LPA_ERR_INVALID_ARG;
  }
}

lpa_status make(lpa_host_graph **out, lpa_host_graph *g) {
  *out = g;
  return LPA_OK;
}

}  // namespace

extern "C" {

lpa_status lpa_hg_generate_road(uint32_t width, uint32_t height, double keep_p, double extra_p, int max_dist,
                                uint64_t seed, lpa_host_graph **out) {
  if (!out || width == 0 || height == 0) return LPA_ERR_INVALID_ARG;
  return guarded([&]() {
    auto *g = new lpa_host_graph();
    lpa::RoadParams p;
    p.width = width;
    p.height = height;
    p.keep_p = keep_p;
    p.extra_p = extra_p;
    p.max_dist = max_dist;
    p.seed = seed;
    try {
      lpa::gen_road(p, g->csr);
    } catch (...) {
      delete g;
      throw;
    }
    g->has_csr = true;
    return make(out, g);
  });
}

lpa_status lpa_hg_generate_rmat(int scale, double edge_factor, double a, double b, double c, uint64_t seed,
                                int bfs_relabel, uint64_t n_limit, lpa_host_graph **out) {
  if (!out) return LPA_ERR_INVALID_ARG;
  return guarded([&]() {
    auto *g = new lpa_host_graph();
    lpa::RmatParams p;
    p.scale = scale;
    p.edge_factor = edge_factor;
    p.a = a;
    p.b = b;
    p.c = c;
    p.seed = seed;
    p.bfs_relabel = bfs_relabel != 0;
    p.n_limit = n_limit;
    try {
      lpa::gen_rmat(p, g->csr);
    } catch (...) {
      delete g;
      throw;
    }
    g->has_csr = true;
    return make(out, g);
  });
}

lpa_status lpa_hg_generate_copy(uint64_t n, uint32_t out_degree, double copy_p, int copy_offset, double zipf_s,
                                uint64_t seed, lpa_host_graph **out) {
  if (!out || out_degree == 0 || out_degree > 64) return LPA_ERR_INVALID_ARG;
  return guarded([&]() {
    auto *g = new lpa_host_graph();
    lpa::CopyParams p;
    p.n = n;
    p.out_degree = out_degree;
    p.copy_p = copy_p;
    p.copy_offset = copy_offset;
    p.zipf_s = zipf_s;
    p.seed = seed;
    try {
      lpa::gen_copy(p, g->csr);
    } catch (...) {
      delete g;
      throw;
    }
    g->has_csr = true;
    return make(out, g);
  });
}

lpa_status lpa_hg_from_csr(uint64_t n, const uint64_t *row, const uint32_t *clm, lpa_host_graph **out) {
  if (!out || !row || (row[n] && !clm)) return LPA_ERR_INVALID_ARG;
  return guarded([&]() {
    auto *g = new lpa_host_graph();
    g->csr.n = n;
    g->csr.row.assign(row, row + n + 1);
    g->csr.clm.assign(clm, clm + row[n]);
    g->has_csr = true;
    return make(out, g);
  });
}

lpa_status lpa_hg_read_edge_list(const char *path, int one_way, lpa_host_graph **out) {
  if (!out || !path) return LPA_ERR_INVALID_ARG;
  return guarded([&]() {
    auto *g = new lpa_host_graph();
    try {
      lpa::read_edge_list(path, one_way != 0, g->csr);
    } catch (...) {
      delete g;
      throw;
    }
    g->has_csr = true;
    return make(out, g);
  });
}

lpa_status lpa_hg_write_edge_list(lpa_host_graph *g, const char *path, int both_arcs) {
  if (!g || !path || !g->has_csr) return LPA_ERR_INVALID_ARG;
  return guarded([&]() {
    lpa::write_edge_list(g->csr, path, both_arcs != 0);
    return LPA_OK;
  });
}

lpa_status lpa_hg_compress(lpa_host_graph *g, int small_thresh, int large_thresh, int threads) {
  if (!g || !g->has_csr) return LPA_ERR_INVALID_ARG;
  return guarded([&]() {
    lpa::CgrParams p;  // (3, 4, 256, 256), src/file.cpp:84
    lpa::cgr_encode(g->csr.view(), p, small_thresh, large_thresh, g->cgr, threads);
    g->has_cgr = true;
    return LPA_OK;
  });
}

lpa_status lpa_hg_compress_gpu(lpa_host_graph *g, int small_thresh, int large_thresh, int device) {
  if (!g || !g->has_csr) return LPA_ERR_INVALID_ARG;
  try {
    lpa::CgrParams p;  // (3, 4, 256, 256), src/file.cpp:84
    lpa::CgrGraph out;
    lpa::cgr_encode_gpu(g->csr.view(), p, small_thresh, large_thresh, out, device);
    g->cgr = std::move(out);
    g->has_cgr = true;
    return LPA_OK;
  } catch (const std::bad_alloc &) {
    return LPA_ERR_OOM;
  } catch (const std::invalid_argument &) {
    return LPA_ERR_INVALID_ARG;
  } catch (const std::exception &) {
    return LPA_ERR_CUDA;  // the device failed (or there is none)
  }
}

lpa_status lpa_hg_load_cgr(const char *base, int small_thresh, lpa_host_graph **out) {
  if (!out || !base) return LPA_ERR_INVALID_ARG;
  return guarded([&]() {
    auto *g = new lpa_host_graph();
    try {
      lpa::cgr_read_files(base, small_thresh, g->cgr);
    } catch (...) {
      delete g;
      throw;
    }
    g->has_cgr = true;
    return make(out, g);
  });
}

lpa_status lpa_hg_write_cgr(lpa_host_graph *g, const char *base) {
  if (!g || !base || !g->has_cgr) return LPA_ERR_INVALID_ARG;
  return guarded([&]() {
    lpa::cgr_write_files(g->cgr, base);
    return LPA_OK;
  });
}

lpa_status lpa_hg_write_csr(lpa_host_graph *g, const char *base) {
  if (!g || !base || !g->has_csr) return LPA_ERR_INVALID_ARG;
  return guarded([&]() {
    lpa::csr_write_files(g->csr, base);
    return LPA_OK;
  });
}

lpa_status lpa_hg_csr(lpa_host_graph *g, uint64_t *n, const uint64_t **row, const uint32_t **clm) {
  if (!g || !g->has_csr) return LPA_ERR_INVALID_ARG;
  if (n) *n = g->csr.n;
  if (row) *row = g->csr.row.data();
  if (clm) *clm = g->csr.clm.data();
  return LPA_OK;
}

lpa_status lpa_hg_desc(lpa_host_graph *g, lpa_graph_desc *d) {
  if (!g || !d || !g->has_cgr) return LPA_ERR_INVALID_ARG;
  const lpa::CgrGraph &c = g->cgr;
  d->num_vertices = c.n;
  d->num_compressed = c.n_c;
  d->words = c.words.data();
  d->num_words = c.words.size();
  d->offsets = c.offsets.data();
  d->vertices = c.vertices.data();
  d->small_graph = c.small_graph.data();
  d->num_small_arcs = c.small_graph.size();
  d->small_offset = c.small_offset.empty() ? nullptr : c.small_offset.data();
  return LPA_OK;
}

lpa_status lpa_hg_concat(const lpa_graph_desc *graphs, size_t num_graphs, lpa_host_graph **out) {
  if (!out) return LPA_ERR_INVALID_ARG;
  *out = nullptr;
  if (!graphs || num_graphs == 0) return LPA_ERR_INVALID_ARG;
  uint64_t n = 0, n_c = 0, bits = 0, arcs = 0;
  for (size_t k = 0; k < num_graphs; k++) {
    const lpa_graph_desc &g = graphs[k];
    if (g.num_compressed > g.num_vertices || (g.num_vertices && !g.vertices)) return LPA_ERR_INVALID_ARG;
    if (g.num_compressed && (!g.words || !g.offsets || g.offsets[0] != 0 ||
                             (g.offsets[g.num_compressed] + 31) / 32 > g.num_words))
      return LPA_ERR_BAD_STREAM;
    if (g.num_vertices > g.num_compressed &&
        (!g.small_offset || g.small_offset[0] != 0 ||
         g.small_offset[g.num_vertices - g.num_compressed] != g.num_small_arcs || (g.num_small_arcs && !g.small_graph)))
      return LPA_ERR_INVALID_ARG;
    n += g.num_vertices;
    n_c += g.num_compressed;
    bits += g.num_compressed ? g.offsets[g.num_compressed] : 0;
    arcs += g.num_vertices > g.num_compressed ? g.num_small_arcs : 0;
  }
  // ids and small-CSR offsets are 32-bit
  if (n > 0xFFFFFFFEull || arcs > 0xFFFFFFFEull) return LPA_ERR_CAPACITY;
  return guarded([&]() -> lpa_status {
    auto *h = new lpa_host_graph();
    lpa::CgrGraph &c = h->cgr;
    c.n = n;
    c.n_c = n_c;
    c.total_bits = bits;
    c.small_thresh = 0;
    c.words.assign((bits + 31) / 32 + 4, 0u);  // + the zero tail
    c.offsets.reserve(n_c + 1);
    c.vertices.resize(n);
    c.small_graph.reserve(arcs);
    if (n > n_c) c.small_offset.reserve(n - n_c + 1);
    uint64_t at = 0, pc = 0, ps = 0, base = 0;
    for (size_t k = 0; k < num_graphs; k++) {
      const lpa_graph_desc &g = graphs[k];
      const uint64_t gb = g.num_compressed ? g.offsets[g.num_compressed] : 0;
      // the graph's bits [0, gb) appended at bit `at` (MSB-first words)
      const uint32_t sh = uint32_t(at & 31);
      for (uint64_t w = 0; w < (gb + 31) / 32; w++) {
        uint32_t x = g.words[w];
        const uint64_t valid = std::min<uint64_t>(32, gb - 32 * w);
        if (valid < 32) x &= ~0u << (32 - valid);  // bits past the graph's end are not its own
        const uint64_t dw = at / 32 + w;
        c.words[dw] |= x >> sh;
        if (sh) c.words[dw + 1] |= x << (32 - sh);
      }
      for (uint64_t i = 0; i < g.num_compressed; i++) c.offsets.push_back(g.offsets[i] + at);
      for (uint64_t i = 0; i < g.num_compressed; i++) c.vertices[pc + i] = uint32_t(g.vertices[i] + base);
      for (uint64_t i = g.num_compressed; i < g.num_vertices; i++)
        c.vertices[n_c + ps + (i - g.num_compressed)] = uint32_t(g.vertices[i] + base);
      if (g.num_vertices > g.num_compressed) {
        const uint32_t ab = uint32_t(c.small_graph.size());
        for (uint64_t i = 0; i < g.num_vertices - g.num_compressed; i++) c.small_offset.push_back(g.small_offset[i] + ab);
        for (uint64_t e = 0; e < g.num_small_arcs; e++) c.small_graph.push_back(uint32_t(g.small_graph[e] + base));
      }
      at += gb;
      pc += g.num_compressed;
      ps += g.num_vertices - g.num_compressed;
      base += g.num_vertices;
    }
    c.offsets.push_back(at);
    if (n > n_c) c.small_offset.push_back(uint32_t(c.small_graph.size()));
    h->has_cgr = true;
    return make(out, h);
  });
}

lpa_status lpa_hg_free(lpa_host_graph *g) {
  if (!g) return LPA_ERR_INVALID_ARG;
  delete g;
  return LPA_OK;
}

}  // extern "C"
