// Fast parallel CGR encoder and the reference's file formats.
//
// The encoder reproduces the reference's CgrCompressor bit for bit
// (src/compressor.cpp:306-515) but works in two parallel passes over a CSR:
// pass 1 measures every vertex's bit length, a prefix sum gives the 64-bit
// offsets, pass 2 writes each vertex's bits at its offset.  The segment
// planner below restates the reference's segment rule, including its two
// quirks that affect the bits:
//   * the overflow test is gamma_size(cnt + 1) + segment_bits + item_bits >
//     seg_len, with item_bits measured on the gap code when the item is not
//     the first of its segment (src/compressor.cpp:390-393, 462);
//   * when a section spills into more than one segment, the final partial
//     segment is not kept: its items are appended, gap-coded, to the last full
//     segment, which is written unpadded (src/compressor.cpp:404-425, 472-484).
#include "lpa/cgr_format.h"

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "parallel.h"

namespace lpa {
namespace {

inline int sig_bit(uint64_t x) {  // floor(log2(x)), x > 0
  return 63 - __builtin_clzll(x);
}
inline uint64_t gamma_size(uint64_t x) { return 2 * uint64_t(sig_bit(x + 1)) + 1; }
inline uint64_t zeta_size(uint64_t x, int k) {
  if (k == 1) return gamma_size(x);
  uint64_t h = uint64_t(sig_bit(x + 1)) / uint64_t(k);
  return (h + 1) * uint64_t(k + 1);
}
inline uint64_t int_2_nat(int64_t x) {  // CgrCompressor::int_2_nat, compressor.h:66-69
  return x >= 0 ? uint64_t(x) << 1 : uint64_t(-((x << 1) + 1));
}

// Counting sink.
struct BitCounter {
  uint64_t bits = 0;
  void zeros(uint64_t n) { bits += n; }
  void put(uint64_t, int len) { bits += uint64_t(len); }
};

// Writing sink over a shared zero-initialised word array.  Words at the two
// ends of this writer's range may be shared with a neighbouring writer and are
// OR-ed atomically.
struct BitWriter {
  uint32_t *words;
  uint64_t pos;
  uint64_t first_word, last_word;
  void or_word(uint64_t w, uint32_t bits) {
    if (!bits) return;
    if (w == first_word || w == last_word)
      __atomic_fetch_or(&words[w], bits, __ATOMIC_RELAXED);
    else
      words[w] |= bits;
  }
  void zeros(uint64_t n) { pos += n; }
  // Writes the low `len` bits of x, MSB first (len <= 64).
  void put(uint64_t x, int len) {
    while (len > 0) {
      uint64_t w = pos >> 5;
      int off = int(pos & 31);
      int take = std::min(32 - off, len);
      uint64_t chunk = (x >> (len - take)) & ((take == 64) ? ~0ull : ((1ull << take) - 1));
      or_word(w, uint32_t(chunk << (32 - off - take)));
      pos += uint64_t(take);
      len -= take;
    }
  }
};

template <class Sink>
inline void put_gamma(Sink &s, uint64_t x) {  // CgrCompressor::encode_gamma
  uint64_t y = x + 1;
  int len = sig_bit(y);
  s.zeros(uint64_t(len));
  s.put(y, len + 1);
}

template <class Sink>
inline void put_zeta(Sink &s, uint64_t x, int k) {  // CgrCompressor::encode_zeta
  if (k == 1) {
    put_gamma(s, x);
    return;
  }
  uint64_t y = x + 1;
  int len = sig_bit(y);
  int h = len / k;
  s.zeros(uint64_t(h));
  s.put(1, 1);
  s.put(y, (h + 1) * k);
}

struct Scratch {
  std::vector<uint32_t> itv_left, itv_len, res;
  std::vector<std::pair<uint64_t, uint64_t>> segs;  // (first item, count)
};

// Plans the segments of one section (item_bits(i, first) gives the bits of
// item i coded as the first of its segment or as a gap).
template <class ItemBits>
void plan_segments(uint64_t n_items, int seg_len, ItemBits item_bits,
                   std::vector<std::pair<uint64_t, uint64_t>> &segs) {
  segs.clear();
  uint64_t cur_bits = 0, cnt = 0, start = 0;
  for (uint64_t i = 0; i < n_items; i++) {
    uint64_t sz = item_bits(i, cnt == 0);
    if (seg_len && gamma_size(cnt + 1) + cur_bits + sz > uint64_t(seg_len)) {
      segs.emplace_back(start, cnt);
      cnt = 0;
      cur_bits = 0;
      start = i;
      sz = item_bits(i, true);
    }
    cnt++;
    cur_bits += sz;
  }
  if (segs.empty())
    segs.emplace_back(start, cnt);
  else
    segs.back().second += cnt;
}

template <class Sink>
void encode_vertex(const uint32_t *nb, uint64_t deg, uint32_t node, const CgrParams &p,
                   Scratch &sc, Sink &s) {
  const int64_t vnode = int64_t(node);
  if (p.res_seg_len == 0) {  // encode_node, src/compressor.cpp:316-323
    put_gamma(s, deg);
    if (deg == 0) return;
  }
  // intervalize (src/compressor.cpp:330-362)
  sc.itv_left.clear();
  sc.itv_len.clear();
  sc.res.clear();
  uint64_t l = 0;
  while (l < deg) {
    uint64_t r = l + 1;
    while (r < deg && uint64_t(nb[r - 1]) + 1 == uint64_t(nb[r])) r++;
    uint64_t len = r - l;
    if (p.min_itv_len != 0 && len >= uint64_t(p.min_itv_len)) {
      sc.itv_left.push_back(nb[l]);
      sc.itv_len.push_back(uint32_t(len));
    } else {
      for (uint64_t i = l; i < r; i++) sc.res.push_back(nb[i]);
    }
    l = r;
  }

  // encode_intervals (src/compressor.cpp:364-439)
  {
    const auto &L = sc.itv_left;
    const auto &N = sc.itv_len;
    auto left_code = [&](uint64_t i, bool first) -> uint64_t {
      if (first) return int_2_nat(int64_t(L[i]) - vnode);
      return uint64_t(int64_t(L[i]) - int64_t(L[i - 1]) - int64_t(N[i - 1]) - 1);
    };
    auto item_bits = [&](uint64_t i, bool first) -> uint64_t {
      return gamma_size(left_code(i, first)) + gamma_size(uint64_t(N[i]) - uint64_t(p.min_itv_len));
    };
    plan_segments(L.size(), p.itv_seg_len, item_bits, sc.segs);
    if (p.itv_seg_len != 0) put_gamma(s, sc.segs.size() - 1);
    for (size_t k = 0; k < sc.segs.size(); k++) {
      uint64_t first = sc.segs[k].first, cnt = sc.segs[k].second;
      bool last = k + 1 == sc.segs.size();
      BitCounter seg_size;
      put_gamma(s, cnt);
      put_gamma(seg_size, cnt);
      for (uint64_t i = first; i < first + cnt; i++) {
        uint64_t lc = left_code(i, i == first);
        uint64_t nc = uint64_t(N[i]) - uint64_t(p.min_itv_len);
        put_gamma(s, lc);
        put_gamma(s, nc);
        seg_size.bits += gamma_size(lc) + gamma_size(nc);
      }
      if (!last && p.itv_seg_len != 0 && seg_size.bits < uint64_t(p.itv_seg_len))
        s.zeros(uint64_t(p.itv_seg_len) - seg_size.bits);
    }
  }

  // encode_residuals (src/compressor.cpp:441-499)
  {
    const auto &R = sc.res;
    auto code = [&](uint64_t i, bool first) -> uint64_t {
      if (first) return int_2_nat(int64_t(R[i]) - vnode);
      return uint64_t(int64_t(R[i]) - int64_t(R[i - 1]) - 1);
    };
    if (p.res_seg_len == 0) {
      for (uint64_t i = 0; i < R.size(); i++) put_zeta(s, code(i, i == 0), p.zeta_k);
      return;
    }
    auto item_bits = [&](uint64_t i, bool first) -> uint64_t {
      return zeta_size(code(i, first), p.zeta_k);
    };
    plan_segments(R.size(), p.res_seg_len, item_bits, sc.segs);
    put_gamma(s, sc.segs.size() - 1);
    for (size_t k = 0; k < sc.segs.size(); k++) {
      uint64_t first = sc.segs[k].first, cnt = sc.segs[k].second;
      bool last = k + 1 == sc.segs.size();
      uint64_t seg_bits = gamma_size(cnt);
      put_gamma(s, cnt);
      for (uint64_t i = first; i < first + cnt; i++) {
        uint64_t c = code(i, i == first);
        put_zeta(s, c, p.zeta_k);
        seg_bits += zeta_size(c, p.zeta_k);
      }
      if (!last && seg_bits < uint64_t(p.res_seg_len)) s.zeros(uint64_t(p.res_seg_len) - seg_bits);
    }
  }
}

void check_params(const CgrParams &p) {
  if (p.zeta_k < 1 || p.zeta_k > 8 || p.min_itv_len < 0 || p.itv_seg_len < 0 || p.res_seg_len < 0)
    throw std::invalid_argument("cgr_encode: unsupported parameters");
}

// ---------------------------------------------------------------- file io --
struct MappedFile {
  void *ptr = nullptr;
  size_t size = 0;
  int fd = -1;
  explicit MappedFile(const std::string &path) {
    fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) throw std::runtime_error("cannot open " + path);
    struct stat st;
    if (fstat(fd, &st) != 0) {
      ::close(fd);
      throw std::runtime_error("cannot stat " + path);
    }
    size = size_t(st.st_size);
    if (size) {
      ptr = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
      if (ptr == MAP_FAILED) {
        ::close(fd);
        throw std::runtime_error("cannot map " + path);
      }
    }
  }
  ~MappedFile() {
    if (ptr && ptr != MAP_FAILED) munmap(ptr, size);
    if (fd >= 0) ::close(fd);
  }
  const char *data() const { return static_cast<const char *>(ptr); }
};

void write_raw(const std::string &path, const void *data, size_t bytes) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) throw std::runtime_error("cannot create " + path);
  if (bytes && std::fwrite(data, 1, bytes, f) != bytes) {
    std::fclose(f);
    throw std::runtime_error("short write " + path);
  }
  std::fclose(f);
}

template <class T>
void read_raw_vec(const std::string &path, std::vector<T> &out) {
  MappedFile mf(path);
  out.resize(mf.size / sizeof(T));
  if (!out.empty()) std::memcpy(out.data(), mf.data(), out.size() * sizeof(T));
}

bool file_exists(const std::string &p) {
  struct stat st;
  return ::stat(p.c_str(), &st) == 0;
}

}  // namespace

uint64_t cgr_vertex_bits(const uint32_t *nbrs, uint64_t deg, uint32_t node, const CgrParams &p) {
  check_params(p);
  Scratch sc;
  BitCounter c;
  encode_vertex(nbrs, deg, node, p, sc, c);
  return c.bits;
}

void cgr_encode(const CsrView &g, const CgrParams &p, int small_thresh, int large_thresh,
                CgrGraph &out, int threads) {
  check_params(p);
  if (small_thresh < 0 || large_thresh < 0 || small_thresh > large_thresh)
    throw std::invalid_argument(
        "cgr_encode: need 0 <= small_thresh <= large_thresh (the reference lists a vertex twice "
        "otherwise)");
  if (g.n > 0xFFFFFFFFull) throw std::invalid_argument("cgr_encode: more than 2^32 vertices");
  threads = resolve_threads(threads);
  const uint64_t n = g.n;
  auto deg = [&](uint64_t v) { return g.row[v + 1] - g.row[v]; };

  // Position order: large by id, mid by id, small by id.
  out = CgrGraph();
  out.n = n;
  out.small_thresh = small_thresh;
  out.large_thresh = large_thresh;
  out.vertices.resize(n);
  {
    uint64_t nl = 0, nm = 0;
    for (uint64_t v = 0; v < n; v++) {
      uint64_t d = deg(v);
      if (d >= uint64_t(large_thresh)) nl++;
      else if (d >= uint64_t(small_thresh)) nm++;
    }
    out.n_large = nl;
    out.n_c = nl + nm;
    uint64_t il = 0, im = nl, is = nl + nm;
    for (uint64_t v = 0; v < n; v++) {
      uint64_t d = deg(v);
      if (d >= uint64_t(large_thresh)) out.vertices[il++] = uint32_t(v);
      else if (d >= uint64_t(small_thresh)) out.vertices[im++] = uint32_t(v);
      else out.vertices[is++] = uint32_t(v);
    }
  }
  const uint64_t n_c = out.n_c;

  // Pass 1: bits per compressed vertex.
  out.offsets.assign(n_c + 1, 0);
  parallel_for(n_c, 4096, threads, [&](uint64_t b, uint64_t e, int) {
    Scratch sc;
    for (uint64_t i = b; i < e; i++) {
      uint32_t v = out.vertices[i];
      BitCounter c;
      encode_vertex(g.clm + g.row[v], deg(v), v, p, sc, c);
      out.offsets[i + 1] = c.bits;
    }
  });
  for (uint64_t i = 0; i < n_c; i++) out.offsets[i + 1] += out.offsets[i];
  out.total_bits = out.offsets[n_c];

  // Pass 2: write.  4 zero words of tail padding for wide device reads.
  const uint64_t nwords = (out.total_bits + 31) / 32;
  out.words.assign(nwords + 4, 0u);
  const uint64_t nchunks = std::max<uint64_t>(1, std::min<uint64_t>(n_c, uint64_t(threads) * 16));
  parallel_for(nchunks, 1, threads, [&](uint64_t cb, uint64_t ce, int) {
    Scratch sc;
    for (uint64_t c = cb; c < ce; c++) {
      uint64_t b = n_c * c / nchunks, e = n_c * (c + 1) / nchunks;
      if (b >= e) continue;
      BitWriter w{out.words.data(), out.offsets[b], out.offsets[b] >> 5,
                  out.offsets[e] == 0 ? 0 : (out.offsets[e] - 1) >> 5};
      for (uint64_t i = b; i < e; i++) {
        uint32_t v = out.vertices[i];
        encode_vertex(g.clm + g.row[v], deg(v), v, p, sc, w);
      }
    }
  });

  // Small CSR (src/compressor.cpp:267-282).
  if (n > n_c) {
    out.small_offset.resize(n - n_c + 1);
    out.small_offset[0] = 0;
    uint64_t acc = 0;
    for (uint64_t i = n_c; i < n; i++) {
      acc += deg(out.vertices[i]);
      if (acc > 0xFFFFFFFFull) throw std::invalid_argument("cgr_encode: small CSR exceeds 2^32 arcs");
      out.small_offset[i - n_c + 1] = uint32_t(acc);
    }
    out.small_graph.resize(acc);
    parallel_for(n - n_c, 8192, threads, [&](uint64_t b, uint64_t e, int) {
      for (uint64_t k = b; k < e; k++) {
        uint32_t v = out.vertices[n_c + k];
        std::memcpy(out.small_graph.data() + out.small_offset[k], g.clm + g.row[v],
                    deg(v) * sizeof(uint32_t));
      }
    });
  }
}

void cgr_write_files(const CgrGraph &g, const std::string &base) {
  // .graph: MSB-first bytes, the last byte zero-padded (src/compressor.cpp:254-263)
  const uint64_t nbytes = (g.total_bits + 7) / 8;
  std::vector<unsigned char> bytes(nbytes);
  for (uint64_t i = 0; i < nbytes; i++) bytes[i] = (unsigned char)(g.words[i >> 2] >> (24 - 8 * (i & 3)));
  write_raw(base + ".graph", bytes.data(), bytes.size());
  // .offset: count, then cumulative end offsets (src/compressor.cpp:190,219,248)
  {
    FILE *f = std::fopen((base + ".offset").c_str(), "w");
    if (!f) throw std::runtime_error("cannot create " + base + ".offset");
    std::string buf;
    buf.reserve(1 << 20);
    char tmp[32];
    int k = std::snprintf(tmp, sizeof(tmp), "%llu\n", (unsigned long long)g.n_c);
    buf.append(tmp, size_t(k));
    for (uint64_t i = 1; i <= g.n_c; i++) {
      k = std::snprintf(tmp, sizeof(tmp), "%llu\n", (unsigned long long)g.offsets[i]);
      buf.append(tmp, size_t(k));
      if (buf.size() > (1u << 20)) {
        std::fwrite(buf.data(), 1, buf.size(), f);
        buf.clear();
      }
    }
    std::fwrite(buf.data(), 1, buf.size(), f);
    std::fclose(f);
  }
  write_raw(base + ".vertices.bin", g.vertices.data(), g.vertices.size() * sizeof(uint32_t));
  if (!g.small_graph.empty()) {
    write_raw(base + ".graph.small.bin", g.small_graph.data(), g.small_graph.size() * sizeof(uint32_t));
    write_raw(base + ".offset.small.bin", g.small_offset.data(),
              g.small_offset.size() * sizeof(uint32_t));
  }
}

void cgr_read_files(const std::string &base, int small_thresh, CgrGraph &out) {
  out = CgrGraph();
  out.small_thresh = small_thresh;
  // .graph (src/file.cpp:197-239)
  {
    MappedFile mf(base + ".graph");
    const unsigned char *b = reinterpret_cast<const unsigned char *>(mf.data());
    uint64_t nwords = (mf.size + 3) / 4;
    out.words.assign(nwords + 4, 0u);
    for (uint64_t i = 0; i < mf.size; i++) out.words[i >> 2] |= uint32_t(b[i]) << (24 - 8 * (i & 3));
  }
  // .offset with 64-bit values (the reference parses them as uint32)
  {
    MappedFile mf(base + ".offset");
    const char *s = mf.data(), *e = s + mf.size;
    auto next = [&](uint64_t &val) -> bool {
      while (s < e && (*s < '0' || *s > '9')) s++;
      if (s >= e) return false;
      uint64_t x = 0;
      while (s < e && *s >= '0' && *s <= '9') x = x * 10 + uint64_t(*s++ - '0');
      val = x;
      return true;
    };
    uint64_t cnt = 0;
    if (!next(cnt)) throw std::runtime_error(base + ".offset: empty");
    out.offsets.resize(cnt + 1);
    out.offsets[0] = 0;
    for (uint64_t i = 1; i <= cnt; i++)
      if (!next(out.offsets[i])) throw std::runtime_error(base + ".offset: truncated");
    for (uint64_t i = 0; i < cnt; i++)
      if (out.offsets[i + 1] < out.offsets[i]) throw std::runtime_error(base + ".offset: not monotone");
    out.n_c = cnt;
    out.total_bits = out.offsets[cnt];
    if (out.total_bits > uint64_t(out.words.size() - 4) * 32)
      throw std::runtime_error(base + ".offset: offsets beyond the end of .graph");
  }
  read_raw_vec(base + ".vertices.bin", out.vertices);
  out.n = out.vertices.size();
  if (out.n < out.n_c) throw std::runtime_error(base + ".vertices.bin: fewer vertices than offsets");
  if (file_exists(base + ".graph.small.bin")) {
    read_raw_vec(base + ".graph.small.bin", out.small_graph);
    read_raw_vec(base + ".offset.small.bin", out.small_offset);
  }
  if (out.n > out.n_c) {
    if (out.small_offset.empty()) out.small_offset.assign(out.n - out.n_c + 1, 0u);
    if (out.small_offset.size() != out.n - out.n_c + 1)
      throw std::runtime_error(base + ".offset.small.bin: size does not match the vertex count");
    if (out.small_offset.back() != out.small_graph.size())
      throw std::runtime_error(base + ".graph.small.bin: size does not match its offsets");
  }
  for (uint32_t v : out.vertices)
    if (v >= out.n) throw std::runtime_error(base + ".vertices.bin: vertex id out of range");
}

void csr_write_files(const CsrGraph &g, const std::string &base) {
  std::vector<uint32_t> row32(g.row.size());
  for (size_t i = 0; i < g.row.size(); i++) {
    if (g.row[i] > 0xFFFFFFFFull) throw std::invalid_argument(".row holds uint32: more than 2^32 arcs");
    row32[i] = uint32_t(g.row[i]);
  }
  write_raw(base + ".row", row32.data(), row32.size() * sizeof(uint32_t));
  write_raw(base + ".clm", g.clm.data(), g.clm.size() * sizeof(uint32_t));
}

void csr_read_files(const std::string &base, CsrGraph &out) {
  std::vector<uint32_t> row32;
  read_raw_vec(base + ".row", row32);
  read_raw_vec(base + ".clm", out.clm);
  if (row32.empty()) throw std::runtime_error(base + ".row: empty");
  out.n = row32.size() - 1;
  out.row.assign(row32.begin(), row32.end());
  if (out.row.back() != out.clm.size()) throw std::runtime_error(base + ".row/.clm: sizes disagree");
}

void read_edge_list(const std::string &path, bool one_way, CsrGraph &out, int threads) {
  threads = resolve_threads(threads);
  MappedFile mf(path);
  const char *base = mf.data();
  const uint64_t size = mf.size;
  // split at line boundaries
  int nt = threads;
  std::vector<uint64_t> cut(nt + 1, size);
  cut[0] = 0;
  for (int t = 1; t < nt; t++) {
    uint64_t c = size * uint64_t(t) / uint64_t(nt);
    while (c < size && base[c] != '\n') c++;
    cut[t] = std::min(size, c + 1);
    if (cut[t] < cut[t - 1]) cut[t] = cut[t - 1];
  }
  std::vector<std::vector<uint32_t>> parts(nt);
  std::vector<uint64_t> maxid(nt, 0);
  std::vector<int> bad(nt, 0);
  parallel_ranges(uint64_t(nt), nt, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t t = b; t < e; t++) {
      const char *s = base + cut[t], *end = base + cut[t + 1];
      auto &vec = parts[t];
      uint64_t mx = 0;
      bool have = false;
      while (s < end) {
        // skip blank space; '#' or '%' comment lines are skipped
        while (s < end && (*s == ' ' || *s == '\t' || *s == '\r' || *s == '\n')) s++;
        if (s >= end) break;
        if (*s == '#' || *s == '%') {
          while (s < end && *s != '\n') s++;
          continue;
        }
        uint64_t x[2];
        for (int k = 0; k < 2; k++) {
          while (s < end && (*s == ' ' || *s == '\t')) s++;
          if (s >= end || *s < '0' || *s > '9') {
            bad[t] = 1;
            s = end;
            break;
          }
          uint64_t val = 0;
          while (s < end && *s >= '0' && *s <= '9') val = val * 10 + uint64_t(*s++ - '0');
          x[k] = val;
        }
        if (bad[t]) break;
        if (x[0] > 0xFFFFFFFEull || x[1] > 0xFFFFFFFEull) {
          bad[t] = 1;
          break;
        }
        vec.push_back(uint32_t(x[0]));
        vec.push_back(uint32_t(x[1]));
        mx = std::max(mx, std::max(x[0], x[1]));
        have = true;
        while (s < end && *s != '\n') s++;
      }
      maxid[t] = have ? mx + 1 : 0;
    }
  });
  for (int t = 0; t < nt; t++)
    if (bad[t]) throw std::runtime_error(path + ": malformed edge list");
  uint64_t n = 0;
  for (int t = 0; t < nt; t++) n = std::max(n, maxid[t]);
  out.n = n;
  std::vector<uint64_t> deg(n + 1, 0);
  for (auto &pv : parts)
    for (size_t i = 0; i < pv.size(); i += 2) {
      deg[pv[i]]++;
      if (one_way) deg[pv[i + 1]]++;
    }
  out.row.assign(n + 1, 0);
  for (uint64_t v = 0; v < n; v++) out.row[v + 1] = out.row[v] + deg[v];
  out.clm.assign(out.row[n], 0);
  std::vector<uint64_t> fill(out.row.begin(), out.row.end() - 1);
  for (auto &pv : parts)
    for (size_t i = 0; i < pv.size(); i += 2) {
      out.clm[fill[pv[i]]++] = pv[i + 1];
      if (one_way) out.clm[fill[pv[i + 1]]++] = pv[i];
    }
  parts.clear();
  parallel_for(n, 4096, threads, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t v = b; v < e; v++) std::sort(out.clm.begin() + out.row[v], out.clm.begin() + out.row[v + 1]);
  });
}

void csr_normalize(CsrGraph &g, bool drop_loops, int threads) {
  const uint64_t n = g.n;
  std::vector<uint64_t> newdeg(n, 0);
  parallel_for(n, 4096, threads, [&](uint64_t b, uint64_t e, int) {
    for (uint64_t v = b; v < e; v++) {
      auto first = g.clm.begin() + g.row[v], last = g.clm.begin() + g.row[v + 1];
      std::sort(first, last);
      auto it = std::unique(first, last);
      if (drop_loops) it = std::remove(first, it, uint32_t(v));
      newdeg[v] = uint64_t(it - first);
    }
  });
  uint64_t acc = 0;
  for (uint64_t v = 0; v < n; v++) {
    uint64_t src = g.row[v];
    g.row[v] = acc;
    if (acc != src) std::memmove(g.clm.data() + acc, g.clm.data() + src, newdeg[v] * sizeof(uint32_t));
    acc += newdeg[v];
  }
  g.row[n] = acc;
  g.clm.resize(acc);
  g.clm.shrink_to_fit();
}

}  // namespace lpa
