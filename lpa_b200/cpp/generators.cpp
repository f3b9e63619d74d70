// Seeded synthetic graph generators (road grid, R-MAT, copy model).
#include "lpa/generators.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "parallel.h"

namespace lpa {
namespace {

// Builds a CSR from per-thread arc lists (u -> v), then sorts and
// de-duplicates every list.
void arcs_to_csr(uint64_t n, std::vector<std::vector<uint64_t>> &parts, CsrGraph &out, int threads,
                 bool drop_loops) {
  out.n = n;
  std::vector<uint64_t> deg(n + 1, 0);
  for (auto &pv : parts)
    for (uint64_t a : pv) deg[a >> 32]++;
  out.row.assign(n + 1, 0);
  for (uint64_t v = 0; v < n; v++) out.row[v + 1] = out.row[v] + deg[v];
  out.clm.assign(out.row[n], 0);
  std::vector<uint64_t> fill(out.row.begin(), out.row.end() - 1);
  for (auto &pv : parts) {
    for (uint64_t a : pv) out.clm[fill[a >> 32]++] = uint32_t(a);
    std::vector<uint64_t>().swap(pv);
  }
  csr_normalize(out, drop_loops, threads);
}

}  // namespace

void gen_road(const RoadParams &p, CsrGraph &out, int threads) {
  threads = resolve_threads(threads);
  const uint64_t W = p.width, H = p.height, n = W * H;
  if (n == 0 || n > 0xFFFFFFFFull) throw std::invalid_argument("gen_road: bad grid size");
  std::vector<std::pair<int, int>> ofs;
  for (int dr = -p.max_dist; dr <= p.max_dist; dr++)
    for (int dc = -p.max_dist; dc <= p.max_dist; dc++) {
      int d = std::abs(dr) + std::abs(dc);
      if (d >= 1 && d <= p.max_dist) ofs.emplace_back(dr, dc);
    }
  const int nt = threads;
  std::vector<std::vector<uint64_t>> parts(nt);
  parallel_ranges(n, nt, [&](uint64_t b, uint64_t e, int t) {
    auto &pv = parts[t];
    auto edge = [&](uint64_t u, uint64_t v) {
      pv.push_back((u << 32) | v);
      pv.push_back((v << 32) | u);
    };
    for (uint64_t v = b; v < e; v++) {
      uint64_t r = v / W, c = v % W;
      Rng rng(p.seed, v);
      double d_right = rng.uniform(), d_down = rng.uniform(), d_extra = rng.uniform();
      uint64_t pick = rng.below(ofs.size());
      if (c + 1 < W && d_right < p.keep_p) edge(v, v + 1);
      if (r + 1 < H && d_down < p.keep_p) edge(v, v + W);
      if (d_extra < p.extra_p && !ofs.empty()) {
        int64_t rr = int64_t(r) + ofs[pick].first, cc = int64_t(c) + ofs[pick].second;
        if (rr >= 0 && rr < int64_t(H) && cc >= 0 && cc < int64_t(W)) edge(v, uint64_t(rr) * W + uint64_t(cc));
      }
    }
  });
  arcs_to_csr(n, parts, out, threads, true);
}

void gen_rmat(const RmatParams &p, CsrGraph &out, int threads) {
  threads = resolve_threads(threads);
  if (p.scale < 1 || p.scale > 31) throw std::invalid_argument("gen_rmat: scale out of range");
  const uint64_t full = 1ull << p.scale;
  const uint64_t n = p.n_limit ? std::min(p.n_limit, full) : full;
  const uint64_t draws = uint64_t(std::llround(p.edge_factor * double(full)));
  const double two32 = 4294967296.0;
  const uint64_t ta = uint64_t(p.a * two32), tb = uint64_t((p.a + p.b) * two32),
                 tc = uint64_t((p.a + p.b + p.c) * two32);
  auto draw = [&](uint64_t i, uint64_t &u, uint64_t &v) {
    Rng rng(p.seed, i);
    uint64_t bits = 0;
    int avail = 0;
    u = v = 0;
    for (int lv = 0; lv < p.scale; lv++) {
      if (!avail) {
        bits = rng.next();
        avail = 2;
      }
      uint64_t x = bits & 0xFFFFFFFFull;
      bits >>= 32;
      avail--;
      uint64_t bu = 0, bv = 0;
      if (x < ta) {
      } else if (x < tb) {
        bv = 1;
      } else if (x < tc) {
        bu = 1;
      } else {
        bu = 1;
        bv = 1;
      }
      u = (u << 1) | bu;
      v = (v << 1) | bv;
    }
  };
  // pass 1: degrees (both directions, loops and out-of-range draws dropped)
  std::vector<uint32_t> deg(n, 0);
  parallel_for(draws, 1 << 16, threads, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t i = b; i < e; i++) {
      uint64_t u, v;
      draw(i, u, v);
      if (u == v || u >= n || v >= n) continue;
      __atomic_fetch_add(&deg[u], 1u, __ATOMIC_RELAXED);
      __atomic_fetch_add(&deg[v], 1u, __ATOMIC_RELAXED);
    }
  });
  CsrGraph g;
  g.n = n;
  g.row.assign(n + 1, 0);
  for (uint64_t v = 0; v < n; v++) g.row[v + 1] = g.row[v] + deg[v];
  std::vector<uint32_t>().swap(deg);
  g.clm.assign(g.row[n], 0);
  std::vector<uint64_t> fill(g.row.begin(), g.row.end() - 1);
  parallel_for(draws, 1 << 16, threads, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t i = b; i < e; i++) {
      uint64_t u, v;
      draw(i, u, v);
      if (u == v || u >= n || v >= n) continue;
      g.clm[__atomic_fetch_add(&fill[u], 1ull, __ATOMIC_RELAXED)] = uint32_t(v);
      g.clm[__atomic_fetch_add(&fill[v], 1ull, __ATOMIC_RELAXED)] = uint32_t(u);
    }
  });
  std::vector<uint64_t>().swap(fill);
  csr_normalize(g, true, threads);
  if (!p.bfs_relabel) {
    out = std::move(g);
    return;
  }
  // BFS relabel
  uint64_t root = 0, best = 0;
  for (uint64_t v = 0; v < n; v++) {
    uint64_t d = g.row[v + 1] - g.row[v];
    if (d > best) {
      best = d;
      root = v;
    }
  }
  std::vector<uint32_t> newid(n, 0xFFFFFFFFu);
  std::vector<uint32_t> queue(n);
  uint64_t head = 0, tail = 0, next_start = 0;
  auto bfs_from = [&](uint64_t s) {
    newid[s] = uint32_t(tail);
    queue[tail++] = uint32_t(s);
    while (head < tail) {
      uint32_t u = queue[head++];
      for (uint64_t k = g.row[u]; k < g.row[u + 1]; k++) {
        uint32_t w = g.clm[k];
        if (newid[w] == 0xFFFFFFFFu) {
          newid[w] = uint32_t(tail);
          queue[tail++] = w;
        }
      }
    }
  };
  if (n) bfs_from(root);
  while (tail < n) {
    while (newid[next_start] != 0xFFFFFFFFu) next_start++;
    bfs_from(next_start);
  }
  out.n = n;
  out.row.assign(n + 1, 0);
  for (uint64_t i = 0; i < n; i++) {
    uint32_t v = queue[i];
    out.row[i + 1] = out.row[i] + (g.row[v + 1] - g.row[v]);
  }
  out.clm.assign(out.row[n], 0);
  parallel_for(n, 4096, threads, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t i = b; i < e; i++) {
      uint32_t v = queue[i];
      uint32_t *dst = out.clm.data() + out.row[i];
      uint64_t d = g.row[v + 1] - g.row[v];
      for (uint64_t k = 0; k < d; k++) dst[k] = newid[g.clm[g.row[v] + k]];
      std::sort(dst, dst + d);
    }
  });
}

void gen_copy(const CopyParams &p, CsrGraph &out, int threads) {
  threads = resolve_threads(threads);
  const uint64_t n = p.n;
  if (n == 0 || n > 0xFFFFFFFFull) throw std::invalid_argument("gen_copy: bad vertex count");
  const uint32_t D = p.out_degree;
  // Zipf(s) rank over [0, n): bounded-Pareto inverse CDF, floor'ed.
  const double s1 = 1.0 - p.zipf_s;
  const double nmax = std::pow(double(n) + 1.0, s1);
  auto zipf = [&](Rng &r) -> uint64_t {
    double u = r.uniform();
    double x = std::pow(1.0 + u * (nmax - 1.0), 1.0 / s1) - 1.0;
    uint64_t k = x < 0 ? 0 : uint64_t(x);
    return k >= n ? n - 1 : k;
  };
  // slot k of v, resolved by following the copy chain (no storage needed)
  auto slot = [&](uint64_t v, uint32_t k) -> uint64_t {
    int64_t add = 0;
    for (;;) {
      Rng r(p.seed, (v << 6) ^ uint64_t(k) ^ 0x5555555555ull);
      double c = r.uniform();
      if (v > 0 && c < p.copy_p) {
        add += int64_t(r.below(uint64_t(2 * p.copy_offset + 1))) - p.copy_offset;
        Rng pr(p.seed, v ^ 0xA5A5A5A5A5A5ull);
        v = pr.below(v);  // prototype: uniform earlier vertex
        continue;
      }
      int64_t t = int64_t(zipf(r)) + add;
      if (t < 0) t = 0;
      if (t >= int64_t(n)) t = int64_t(n) - 1;
      return uint64_t(t);
    }
  };
  CsrGraph g;
  g.n = n;
  g.row.resize(n + 1);
  for (uint64_t v = 0; v <= n; v++) g.row[v] = v * D;
  g.clm.assign(n * D, 0);
  parallel_for(n, 1 << 14, threads, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t v = b; v < e; v++)
      for (uint32_t k = 0; k < D; k++) g.clm[v * D + k] = uint32_t(slot(v, k));
  });
  csr_normalize(g, true, threads);
  out = std::move(g);
}

void csr_edges_once(const CsrGraph &g, std::vector<std::pair<uint32_t, uint32_t>> &edges) {
  edges.clear();
  for (uint64_t u = 0; u < g.n; u++)
    for (uint64_t k = g.row[u]; k < g.row[u + 1]; k++)
      if (uint64_t(g.clm[k]) >= u) edges.emplace_back(uint32_t(u), g.clm[k]);
}

void write_edge_list(const CsrGraph &g, const std::string &path, bool both_arcs) {
  FILE *f = std::fopen(path.c_str(), "w");
  if (!f) throw std::runtime_error("cannot create " + path);
  std::string buf;
  char tmp[48];
  for (uint64_t u = 0; u < g.n; u++)
    for (uint64_t k = g.row[u]; k < g.row[u + 1]; k++) {
      if (!both_arcs && uint64_t(g.clm[k]) < u) continue;
      int len = std::snprintf(tmp, sizeof(tmp), "%llu %u\n", (unsigned long long)u, g.clm[k]);
      buf.append(tmp, size_t(len));
      if (buf.size() > (1u << 20)) {
        std::fwrite(buf.data(), 1, buf.size(), f);
        buf.clear();
      }
    }
  std::fwrite(buf.data(), 1, buf.size(), f);
  std::fclose(f);
}

}  // namespace lpa
