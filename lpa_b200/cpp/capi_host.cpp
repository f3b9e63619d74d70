// C ABI of the host format layer (lpa_hg_*): generators, the fast
// bit-identical CGR encoder and the reference's file formats.
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

lpa_status lpa_hg_free(lpa_host_graph *g) {
  if (!g) return LPA_ERR_INVALID_ARG;
  delete g;
  return LPA_OK;
}

}  // extern "C"
