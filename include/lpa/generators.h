// Seeded synthetic graph generators standing in for the reference's datasets
// (roadNet-CA, LiveJournal, uk-2002, ... are not available).  Every generator
// is deterministic for a given seed and thread count independent: each random
// decision is drawn from a counter-based stream keyed by (seed, item).
#pragma once
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "lpa/cgr_format.h"

namespace lpa {

// Road-like planar graph: a width x height grid in row-major ids; each
// 4-neighbour edge is kept with probability keep_p; each vertex, with
// probability extra_p, adds one edge to a uniformly chosen other vertex within
// Manhattan distance <= max_dist (offsets leaving the grid add nothing).
struct RoadParams {
  uint32_t width = 362, height = 362;
  double keep_p = 0.7;
  double extra_p = 0.02;
  int max_dist = 3;
  uint64_t seed = 1;
};

// R-MAT: edge_factor * 2^scale draws with quadrant probabilities (a, b, c,
// 1-a-b-c); self loops dropped, symmetrised, de-duplicated.  With
// bfs_relabel, ids are reassigned in BFS order from the highest-degree vertex
// (lowest id on ties; neighbours visited in ascending id; unreached vertices
// continue from the lowest unvisited id).  When n_limit > 0, draws with an
// endpoint >= n_limit are discarded and n = n_limit, else n = 2^scale.
struct RmatParams {
  int scale = 24;
  double edge_factor = 16.0;
  double a = 0.57, b = 0.19, c = 0.19;
  uint64_t seed = 1;
  bool bfs_relabel = true;
  uint64_t n_limit = 0;
};

// Copy model (web-like): vertex v (v > 0) picks a uniform prototype u < v;
// each of its `out_degree` slots copies the prototype's slot (plus a uniform
// offset in [-copy_offset, copy_offset], clipped) with probability copy_p,
// otherwise draws a Zipf(zipf_s) target.  Lists sorted, de-duplicated,
// loops dropped.  Directed (out-lists only).
struct CopyParams {
  uint64_t n = 100000000ull;
  uint32_t out_degree = 30;
  double copy_p = 0.6;
  int copy_offset = 8;
  double zipf_s = 1.1;
  uint64_t seed = 1;
};

void gen_road(const RoadParams &p, CsrGraph &out, int threads = 0);
void gen_rmat(const RmatParams &p, CsrGraph &out, int threads = 0);
void gen_copy(const CopyParams &p, CsrGraph &out, int threads = 0);

// Undirected edges of a symmetric CSR, each once with u < v (loops once).
void csr_edges_once(const CsrGraph &g, std::vector<std::pair<uint32_t, uint32_t>> &edges);
// Writes "u v" lines: every arc (both directions) when both_arcs, else each
// undirected edge once (u <= v).
void write_edge_list(const CsrGraph &g, const std::string &path, bool both_arcs);

// Counter-based random stream (splitmix64 finaliser over (seed, key, ctr)).
struct Rng {
  uint64_t s;
  static uint64_t mix(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  }
  Rng(uint64_t seed, uint64_t key) : s(mix(mix(seed) ^ (key * 0xd1b54a32d192ed03ull))) {}
  uint64_t next() { return mix(s += 0x9e3779b97f4a7c15ull); }
  double uniform() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
  uint64_t below(uint64_t n) { return n ? uint64_t((unsigned __int128)next() * n >> 64) : 0; }
};

}  // namespace lpa
