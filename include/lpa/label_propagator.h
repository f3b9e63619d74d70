// LabelPropagator: the reference's propagator interface
// (include/label_propagator.h:11-52) and B200Propagator, the sm_100a
// implementation behind it (in the role of NovaPlusPropagator,
// baselines/novaplus/novaplus_propogator.cuh:24-199), calling the C ABI.
#pragma once
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "lpa/graph.h"
#include "lpa_capi.h"

namespace lpa {

class Timer {  // include/utils.h:19-42 (wall clock, milliseconds)
 public:
  void start() { t0_ = std::chrono::steady_clock::now(); }
  void stop() { t1_ = std::chrono::steady_clock::now(); }
  double elapsed_time() const { return std::chrono::duration<double, std::milli>(t1_ - t0_).count(); }
  double elapsed_second() const { return elapsed_time() / 1e3; }

 private:
  std::chrono::steady_clock::time_point t0_, t1_;
};

template <typename V, typename E>
class LabelPropagator {
 public:
  using GraphT = CSRGraph<V, E>;
  using CGRGraphT = CGRGraph<V, E>;
  using CGRGraphTPure = CGRGraphPure<V, E>;
  using CommonGraph = Graph<V, E>;
  LabelPropagator() = default;
  explicit LabelPropagator(int n) : n_(n), labels(new V[n]) {}
  virtual ~LabelPropagator() = default;

  // Runs niter iterations; returns (LP milliseconds, preprocess + LP milliseconds).
  virtual std::pair<double, double> run(int niter) = 0;

  std::vector<V> get_labels() {
    auto p = labels.get();
    return std::vector<V>(p, p + n_);
  }

 protected:
  int n_ = 0;

 public:
  std::unique_ptr<V[]> labels;
};

struct PropagatorOptions {
  uint32_t cms_threshold = 128;  // include/decoder.cuh:51 (THREADS_NUM)
  uint64_t cms_seed = 1;
  int dispatch = LPA_DISPATCH_FIXED;
  int force_variant = LPA_VARIANT_BLOCK;
  bool early_exit = false;
  bool print_iterations = true;  // "%d: %f (ms), updated %d" per iteration
  int device = 0;
};

// The B200 propagator over a CGRGraph.  Throws std::runtime_error when the
// library reports an error (there is no CPU fallback).
template <typename V, typename E>
class B200Propagator : public LabelPropagator<V, E> {
 public:
  using CGRGraphT = CGRGraph<V, E>;
  explicit B200Propagator(std::shared_ptr<CGRGraphT> _G, PropagatorOptions o = PropagatorOptions())
      : LabelPropagator<V, E>(int(_G->n)), G(std::move(_G)), opts(o) {}
  ~B200Propagator() override {
    if (h_) lpa_destroy(h_);
  }

  std::pair<double, double> run(int niter) override {
    Timer t_all, t_lp;
    t_all.start();
    preprocess();
    throw_if(lpa_init_labels(h_), "lpa_init_labels");
    t_lp.start();
    if (opts.print_iterations && !opts.early_exit) {
      for (int i = 0; i < niter; i++) {
        Timer t;
        t.start();
        uint64_t changed = 0;
        throw_if(lpa_iterate(h_, &changed), "lpa_iterate");
        t.stop();
        std::printf("%d: %f (ms), updated %d\n", i + 1, t.elapsed_time(), int(changed));
      }
    } else {
      int done = 0;
      throw_if(lpa_run(h_, niter, opts.early_exit ? 1 : 0, &done), "lpa_run");
      iterations_done = done;
      if (opts.print_iterations) {
        std::vector<uint64_t> hist(static_cast<size_t>(done));
        throw_if(lpa_get_changed_history(h_, hist.data(), hist.size()), "history");
        for (int i = 0; i < done; i++) std::printf("%d: - (ms), updated %d\n", i + 1, int(hist[size_t(i)]));
      }
    }
    throw_if(lpa_get_labels(h_, reinterpret_cast<uint32_t *>(this->labels.get()), size_t(G->n)), "lpa_get_labels");
    t_lp.stop();
    t_all.stop();
    return {t_lp.elapsed_time(), t_all.elapsed_time()};
  }

  // Copies the graph to the device and builds the plan (once).
  void preprocess() {
    if (h_) return;
    lpa_graph_desc d{};
    d.num_vertices = G->vertices.size();
    d.num_compressed = G->cgr_offsets.empty() ? 0 : G->cgr_offsets.size() - 1;
    d.words = reinterpret_cast<const uint32_t *>(G->cgr_neighbors.data());
    d.num_words = G->cgr_neighbors.size();
    d.offsets = G->cgr_offsets.data();
    d.vertices = reinterpret_cast<const uint32_t *>(G->vertices.data());
    d.small_graph = reinterpret_cast<const uint32_t *>(G->csr_small_neighbors.data());
    d.num_small_arcs = G->csr_small_neighbors.size();
    d.small_offset = G->csr_small_offsets.empty() ? nullptr
                                                  : reinterpret_cast<const uint32_t *>(G->csr_small_offsets.data());
    lpa_opts o;
    lpa_opts_default(&o);
    o.device = opts.device;
    o.cms_threshold = opts.cms_threshold;
    o.cms_seed = opts.cms_seed;
    o.dispatch = opts.dispatch;
    o.force_variant = opts.force_variant;
    throw_if(lpa_create(&d, &o, &h_), "lpa_create");
  }

  lpa_handle *handle() { return h_; }
  int iterations_done = 0;
  std::shared_ptr<CGRGraphT> G;
  PropagatorOptions opts;

 private:
  struct lpa_handle *h_ = nullptr;
  void throw_if(lpa_status st, const char *what) {
    if (st != LPA_OK)
      throw std::runtime_error(std::string(what) + ": " + lpa_status_str(st) +
                               (h_ ? std::string(" (") + lpa_last_error(h_) + ")" : std::string()));
  }
};

}  // namespace lpa
