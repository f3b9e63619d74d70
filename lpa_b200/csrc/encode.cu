// GPU-side CGR encoder, byte-identical to lpa::cgr_encode (cgr_format.cpp),
// which restates the reference's CgrCompressor (src/compressor.cpp:306-515).
//
// The host keeps the cheap O(n) parts (position order, prefix sum of the bit
// lengths, small CSR); the device does the per-vertex work, one thread per
// compressed position:
//   pass 1  walks the neighbour list once and plans both sections' 256-bit
//           segments with the reference's rule (a segment closes when
//           gamma(cnt + 1) + its bits + the next item's bits exceed 256; the
//           final partial segment joins the last closed one, unpadded), giving
//           the vertex's bit length, its segment counts and the interval
//           section's length;
//   pass 2  plans again and writes each segment once the next one has closed
//           (so it is known not to be the last), re-reading its items from
//           the neighbour list: no per-thread item buffers.  Non-last segments
//           sit at fixed 256-bit steps, so every segment's position is known.
// Words shared with the neighbouring vertices are OR-ed atomically into a
// zeroed stream.  Only the reference's parameters (zeta k = 3, intervals of
// >= 4, 256-bit segments for both sections) are supported.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "lpa/cgr_format.h"

namespace {

constexpr uint32_t kSegLen = 256;
constexpr uint32_t kMinItv = 4;

__device__ __forceinline__ int sig_bit(uint64_t x) { return 63 - __clzll(x); }  // x > 0
__device__ __forceinline__ uint32_t gamma_size(uint64_t x) { return 2u * uint32_t(sig_bit(x + 1)) + 1u; }
__device__ __forceinline__ uint32_t zeta3_size(uint64_t x) { return (uint32_t(sig_bit(x + 1)) / 3u + 1u) * 4u; }
__device__ __forceinline__ uint64_t int_2_nat(int64_t x) {
  return x >= 0 ? uint64_t(x) << 1 : uint64_t(-((x << 1) + 1));
}

// Items of one section in neighbour order: intervals (maximal runs of >= 4
// consecutive ids: left, len) or residuals (the other ids one by one).  idx is
// where a later scan restarts to yield this item first: an interval's run
// start, or a residual's own index (a run entered in its middle is shorter,
// so still residual).
struct Scan {
  const uint32_t *nb;
  uint64_t deg, k, rk, re;
  bool itv;
  __device__ Scan(const uint32_t *nb_, uint64_t deg_, uint64_t k0, bool itv_)
      : nb(nb_), deg(deg_), k(k0), rk(0), re(0), itv(itv_) {}
  __device__ bool next(uint32_t &a, uint32_t &len, uint64_t &idx) {
    for (;;) {
      if (rk < re) {
        idx = rk;
        a = nb[rk++];
        len = 1;
        return true;
      }
      if (k >= deg) return false;
      const uint64_t l = k;
      uint64_t r = l + 1;
      while (r < deg && uint64_t(nb[r - 1]) + 1 == uint64_t(nb[r])) r++;
      k = r;
      if (r - l >= kMinItv) {
        if (itv) {
          idx = l;
          a = nb[l];
          len = uint32_t(r - l);
          return true;
        }
      } else if (!itv) {
        rk = l;
        re = r;
      }
    }
  }
};

// Code values of an item: first of its segment (relative to the node) or a
// gap from the previous item of the section.
struct Codes {
  uint64_t first, gap;
};
__device__ __forceinline__ Codes item_codes(bool itv, uint32_t a, uint32_t len, uint32_t pa, uint32_t plen,
                                            uint32_t node, bool has_prev) {
  Codes c;
  c.first = int_2_nat(int64_t(a) - int64_t(node));
  if (!has_prev) c.gap = 0;
  else if (itv) c.gap = uint64_t(int64_t(a) - int64_t(pa) - int64_t(plen) - 1);
  else c.gap = uint64_t(int64_t(a) - int64_t(pa) - 1);
  return c;
}
__device__ __forceinline__ uint32_t item_bits(bool itv, uint64_t code, uint32_t len) {
  return itv ? gamma_size(code) + gamma_size(uint64_t(len) - kMinItv) : zeta3_size(code);
}

// plan_segments (cgr_format.cpp) as a stream.  close(start, cnt) is called
// for every segment the rule closes.
struct Plan {
  uint32_t cnt = 0, nclosed = 0, last_cnt = 0;
  uint64_t cur = 0, start = 0, last_bits = 0, tail_gap = 0;
  template <class Close>
  __device__ void feed(uint32_t fs, uint32_t gs, uint64_t idx, Close &&close) {
    uint32_t sz = cnt == 0 ? fs : gs;
    if (gamma_size(uint64_t(cnt) + 1) + cur + sz > kSegLen) {
      close(start, cnt);
      last_cnt = cnt;
      last_bits = gamma_size(cnt) + cur;
      nclosed++;
      cnt = 0;
      cur = 0;
      tail_gap = 0;
      sz = fs;
    }
    if (cnt == 0) start = idx;
    cnt++;
    cur += sz;
    tail_gap += gs;
  }
  __device__ uint32_t nseg() const { return nclosed ? nclosed : 1u; }
  // section bits after its header: 256 per non-last segment, then the last
  // (the last closed one with the tail's items appended as gaps)
  __device__ uint64_t bits() const {
    if (nclosed == 0) return gamma_size(cnt) + cur;
    return uint64_t(nclosed - 1) * kSegLen + gamma_size(uint64_t(last_cnt) + cnt) + (last_bits - gamma_size(last_cnt)) +
           tail_gap;
  }
};

// Plans one section over the neighbour list; close is forwarded.
template <class Close>
__device__ Plan plan_section(const uint32_t *nb, uint64_t deg, uint32_t node, bool itv, Close &&close) {
  Plan pl;
  Scan sc(nb, deg, 0, itv);
  uint32_t a, len, pa = 0, plen = 0;
  uint64_t idx;
  bool has_prev = false;
  while (sc.next(a, len, idx)) {
    const Codes c = item_codes(itv, a, len, pa, plen, node, has_prev);
    pl.feed(item_bits(itv, c.first, len), has_prev ? item_bits(itv, c.gap, len) : 0u, idx, close);
    pa = a;
    plen = len;
    has_prev = true;
  }
  return pl;
}

// MSB-first bit writer into a zeroed word array; each word is OR-ed once,
// atomically (the first and last words of a vertex are shared).
struct Writer {
  uint32_t *w;
  uint64_t nwords;  // words outside the stream are never touched (bad is set)
  uint64_t pos;
  uint64_t word;
  uint32_t acc;
  bool has, bad;
  __device__ void flush() {
    if (has && acc) {
      if (word < nwords) atomicOr(w + word, acc);
      else bad = true;
    }
    has = false;
  }
  __device__ void emit(uint64_t wi, uint32_t bits) {
    if (has && wi == word) {
      acc |= bits;
      return;
    }
    flush();
    word = wi;
    acc = bits;
    has = true;
  }
  __device__ void put(uint64_t x, int len) {  // the low len (<= 64) bits of x
    while (len > 0) {
      const uint64_t wi = pos >> 5;
      const int off = int(pos & 31);
      const int take = min(32 - off, len);
      const uint64_t chunk = (x >> (len - take)) & ((1ull << take) - 1);
      emit(wi, uint32_t(chunk << (32 - off - take)));
      pos += uint64_t(take);
      len -= take;
    }
  }
  __device__ void gamma(uint64_t x) {
    const uint64_t y = x + 1;
    const int len = sig_bit(y);
    pos += uint64_t(len);
    put(y, len + 1);
  }
  __device__ void zeta3(uint64_t x) {
    const uint64_t y = x + 1;
    const int h = sig_bit(y) / 3;
    pos += uint64_t(h);
    put(1, 1);
    put(y, (h + 1) * 3);
  }
};

// Writes the segment of cnt items starting at scan index start at position
// at: gamma(cnt), the first item coded against the node, the rest as gaps.
__device__ void write_segment(Writer &wr, uint64_t at, const uint32_t *nb, uint64_t deg, uint32_t node, bool itv,
                              uint64_t start, uint32_t cnt) {
  wr.pos = at;
  wr.gamma(cnt);
  Scan sc(nb, deg, start, itv);
  uint32_t a, len, pa = 0, plen = 0;
  uint64_t idx;
  for (uint32_t i = 0; i < cnt && sc.next(a, len, idx); i++) {
    const Codes c = item_codes(itv, a, len, pa, plen, node, i > 0);
    const uint64_t code = i == 0 ? c.first : c.gap;
    if (itv) {
      wr.gamma(code);
      wr.gamma(uint64_t(len) - kMinItv);
    } else {
      wr.zeta3(code);
    }
    pa = a;
    plen = len;
  }
}

// One section: plan it again, writing every closed segment once the next one
// closes, then the last (merged with the tail) at the end.
__device__ void write_section(Writer &wr, uint64_t base, const uint32_t *nb, uint64_t deg, uint32_t node, bool itv) {
  bool pend = false;
  uint64_t pstart = 0;
  uint32_t pcnt = 0, pindex = 0, closed = 0;
  const Plan pl = plan_section(nb, deg, node, itv, [&](uint64_t start, uint32_t cnt) {
    if (pend) write_segment(wr, base + uint64_t(pindex) * kSegLen, nb, deg, node, itv, pstart, pcnt);
    pend = true;
    pstart = start;
    pcnt = cnt;
    pindex = closed++;
  });
  if (pend) write_segment(wr, base + uint64_t(pindex) * kSegLen, nb, deg, node, itv, pstart, pcnt + pl.cnt);
  else write_segment(wr, base, nb, deg, node, itv, pl.start, pl.cnt);
}

struct NoClose {
  __device__ void operator()(uint64_t, uint32_t) const {}
};

// Pass 1: per compressed position, its bit length and the numbers pass 2
// needs (segment counts, interval section length after its header).
__global__ void k_encode_size(const uint64_t *row, const uint32_t *clm, const uint32_t *vertices, uint64_t n_c,
                              uint64_t *bits, uint32_t *nseg_i, uint32_t *nseg_r, uint64_t *itv_bits, uint32_t *err) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n_c; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t v = vertices[i];
    const uint32_t *nb = clm + row[v];
    const uint64_t deg = row[v + 1] - row[v];
    for (uint64_t k = 1; k < deg; k++)
      if (nb[k] <= nb[k - 1]) {  // the gap codes need strictly ascending lists
        atomicOr(err, 1u);
        break;
      }
    const Plan pi = plan_section(nb, deg, v, true, NoClose{});
    const Plan pr = plan_section(nb, deg, v, false, NoClose{});
    nseg_i[i] = pi.nseg();
    nseg_r[i] = pr.nseg();
    itv_bits[i] = pi.bits();
    bits[i] = gamma_size(pi.nseg() - 1) + pi.bits() + gamma_size(pr.nseg() - 1) + pr.bits();
  }
}

// Pass 2: writes every compressed position at its offset.
__global__ void k_encode_write(const uint64_t *row, const uint32_t *clm, const uint32_t *vertices, uint64_t n_c,
                               const uint64_t *offsets, const uint32_t *nseg_i, const uint32_t *nseg_r,
                               const uint64_t *itv_bits, uint32_t *words, uint64_t nwords, uint32_t *err) {
  for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n_c; i += uint64_t(gridDim.x) * blockDim.x) {
    const uint32_t v = vertices[i];
    const uint32_t *nb = clm + row[v];
    const uint64_t deg = row[v + 1] - row[v];
    Writer wr{words, nwords, offsets[i], 0, 0, false, false};
    wr.gamma(nseg_i[i] - 1);
    const uint64_t ibase = wr.pos;
    write_section(wr, ibase, nb, deg, v, true);
    wr.pos = ibase + itv_bits[i];
    wr.gamma(nseg_r[i] - 1);
    const uint64_t rbase = wr.pos;
    write_section(wr, rbase, nb, deg, v, false);
    wr.flush();
    if (wr.bad || wr.pos != offsets[i + 1]) atomicOr(err, 2u);
  }
}

// The small CSR: one warp copies each small vertex's list (lists are
// contiguous in both arrays, positions n_c.. in order).
__global__ void k_gather_small(const uint64_t *row, const uint32_t *clm, const uint32_t *vertices_small,
                               const uint32_t *small_off, uint64_t ns, uint32_t *small_graph) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t nw = (uint64_t(gridDim.x) * blockDim.x) >> 5;
  for (uint64_t k = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5; k < ns; k += nw) {
    const uint32_t v = vertices_small[k];
    const uint64_t b = row[v], d = row[v + 1] - b;
    uint32_t *dst = small_graph + small_off[k];
    for (uint64_t j = lane; j < d; j += 32) dst[j] = clm[b + j];
  }
}

void ck(cudaError_t e, const char *what) {
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw std::runtime_error(std::string("cgr_encode_gpu: ") + what + ": " + cudaGetErrorString(e));
  }
}

template <class T>
struct DevBuf {
  T *p = nullptr;
  explicit DevBuf(size_t n) { ck(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc"); }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
};

}  // namespace

namespace lpa {

void cgr_encode_gpu(const CsrView &g, const CgrParams &p, int small_thresh, int large_thresh, CgrGraph &out,
                    int device) {
  if (p.zeta_k != 3 || p.min_itv_len != int(kMinItv) || p.itv_seg_len != int(kSegLen) ||
      p.res_seg_len != int(kSegLen))
    throw std::invalid_argument("cgr_encode_gpu: only the reference parameters (3, 4, 256, 256)");
  if (small_thresh < 0 || large_thresh < 0 || small_thresh > large_thresh)
    throw std::invalid_argument("cgr_encode_gpu: need 0 <= small_thresh <= large_thresh");
  if (g.n > 0xFFFFFFFFull) throw std::invalid_argument("cgr_encode_gpu: more than 2^32 vertices");
  ck(cudaSetDevice(device), "cudaSetDevice");
  const uint64_t n = g.n, m = n ? g.row[n] : 0;
  auto deg = [&](uint64_t v) { return g.row[v + 1] - g.row[v]; };

  // position order: large by id, mid by id, small by id (as the host encoder)
  out = CgrGraph();
  out.n = n;
  out.small_thresh = small_thresh;
  out.large_thresh = large_thresh;
  out.vertices.resize(n);
  uint64_t nl = 0, nm = 0;
  for (uint64_t v = 0; v < n; v++) {
    const uint64_t d = deg(v);
    if (d >= uint64_t(large_thresh)) nl++;
    else if (d >= uint64_t(small_thresh)) nm++;
  }
  out.n_large = nl;
  out.n_c = nl + nm;
  {
    uint64_t il = 0, im = nl, is = nl + nm;
    for (uint64_t v = 0; v < n; v++) {
      const uint64_t d = deg(v);
      if (d >= uint64_t(large_thresh)) out.vertices[il++] = uint32_t(v);
      else if (d >= uint64_t(small_thresh)) out.vertices[im++] = uint32_t(v);
      else out.vertices[is++] = uint32_t(v);
    }
  }
  const uint64_t n_c = out.n_c;
  out.offsets.assign(n_c + 1, 0);

  // the CSR on the device, once, for both the encoder and the small CSR
  DevBuf<uint64_t> d_row(n + 1);
  DevBuf<uint32_t> d_clm(m);
  ck(cudaMemcpy(d_row.p, g.row, (n + 1) * 8, cudaMemcpyHostToDevice), "upload row");
  if (m) ck(cudaMemcpy(d_clm.p, g.clm, m * 4, cudaMemcpyHostToDevice), "upload clm");
  int sms = 148;
  ck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "attribute");
  if (n_c) {
    DevBuf<uint64_t> d_bits(n_c), d_itv(n_c), d_off(n_c + 1);
    DevBuf<uint32_t> d_vert(n_c), d_nsi(n_c), d_nsr(n_c), d_err(1);
    ck(cudaMemcpy(d_vert.p, out.vertices.data(), n_c * 4, cudaMemcpyHostToDevice), "upload positions");
    ck(cudaMemset(d_err.p, 0, 4), "clear error");
    const int threads = 128;
    const int blocks = int(std::min<uint64_t>((n_c + threads - 1) / threads, uint64_t(sms) * 16));
    k_encode_size<<<blocks, threads>>>(d_row.p, d_clm.p, d_vert.p, n_c, d_bits.p, d_nsi.p, d_nsr.p, d_itv.p, d_err.p);
    ck(cudaGetLastError(), "size pass");
    std::vector<uint64_t> bits(n_c);
    ck(cudaMemcpy(bits.data(), d_bits.p, n_c * 8, cudaMemcpyDeviceToHost), "read sizes");
    uint32_t err = 0;
    ck(cudaMemcpy(&err, d_err.p, 4, cudaMemcpyDeviceToHost), "read error");
    if (err) throw std::invalid_argument("cgr_encode_gpu: neighbour lists must be strictly ascending");
    for (uint64_t i = 0; i < n_c; i++) out.offsets[i + 1] = out.offsets[i] + bits[i];
    out.total_bits = out.offsets[n_c];
    const uint64_t nwords = (out.total_bits + 31) / 32 + 4;  // 4 zero words of tail, as the host encoder
    DevBuf<uint32_t> d_words(nwords);
    ck(cudaMemset(d_words.p, 0, nwords * 4), "clear stream");
    ck(cudaMemcpy(d_off.p, out.offsets.data(), (n_c + 1) * 8, cudaMemcpyHostToDevice), "upload offsets");
    k_encode_write<<<blocks, threads>>>(d_row.p, d_clm.p, d_vert.p, n_c, d_off.p, d_nsi.p, d_nsr.p, d_itv.p,
                                        d_words.p, nwords, d_err.p);
    ck(cudaGetLastError(), "write pass");
    ck(cudaMemcpy(&err, d_err.p, 4, cudaMemcpyDeviceToHost), "read error");
    if (err) throw std::runtime_error("cgr_encode_gpu: a vertex's bits did not end at its offset");
    out.words.resize(nwords);
    ck(cudaMemcpy(out.words.data(), d_words.p, nwords * 4, cudaMemcpyDeviceToHost), "read stream");
  } else {
    out.total_bits = 0;
    out.words.assign(4, 0u);
  }

  // small CSR (src/compressor.cpp:267-282): offsets on the host, the gather
  // of the lists on the device
  if (n > n_c) {
    const uint64_t ns = n - n_c;
    out.small_offset.resize(ns + 1);
    out.small_offset[0] = 0;
    uint64_t acc = 0;
    for (uint64_t i = n_c; i < n; i++) {
      acc += deg(out.vertices[i]);
      if (acc > 0xFFFFFFFFull) throw std::invalid_argument("cgr_encode_gpu: small CSR exceeds 2^32 arcs");
      out.small_offset[i - n_c + 1] = uint32_t(acc);
    }
    out.small_graph.resize(acc);
    if (acc) {
      DevBuf<uint32_t> d_vs(ns), d_so(ns + 1), d_sg(acc);
      ck(cudaMemcpy(d_vs.p, out.vertices.data() + n_c, ns * 4, cudaMemcpyHostToDevice), "upload small positions");
      ck(cudaMemcpy(d_so.p, out.small_offset.data(), (ns + 1) * 4, cudaMemcpyHostToDevice), "upload small offsets");
      k_gather_small<<<sms * 8, 256>>>(d_row.p, d_clm.p, d_vs.p, d_so.p, ns, d_sg.p);
      ck(cudaGetLastError(), "small CSR gather");
      ck(cudaMemcpy(out.small_graph.data(), d_sg.p, acc * 4, cudaMemcpyDeviceToHost), "read small CSR");
    }
  }
}

}  // namespace lpa
