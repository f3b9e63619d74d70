// Device-side CGR decode primitives and shared helpers (sm_100a).
//
// The bit reader restates the reference's CgrReader (include/graph_utils.cuh:
// 19-98) with 64-bit bit positions and a 64-bit window, so one window serves
// any gamma code (<= 63 bits) or zeta_3 code (<= 44 bits) of a 32-bit value.
// Every read position is checked against the vertex's bit range by the
// callers; a violation sets the device error word (never traps).
#pragma once
#include <cstdint>
#include <type_traits>
#include <cuda_runtime.h>

namespace lpa_dev {

constexpr uint32_t kFull = 0xFFFFFFFFu;
constexpr uint32_t kSegBits = 256;  // INTERVAL_SEGMENT_LEN, graph_utils.cuh:17
constexpr uint32_t kMinItv = 4;     // minimum interval length, graph_utils.cuh:172
constexpr int kCmsDepth = 4;
constexpr uint32_t kCmsWidth = 1024;

// device error word values (first error wins)
enum : uint32_t {
  kErrNone = 0,
  kErrBadStream = 1,  // a decode left the vertex's bit range or produced an id >= n
  kErrCapacity = 2,   // more items than a staging buffer was planned for
  kErrTimeout = 3,    // a bounded wait gave up
};

__device__ __forceinline__ void set_error(uint32_t *err, uint32_t code) {
  if (err) atomicCAS(err, kErrNone, code);
}

// Bitstream and mixed-graph arrays as the kernels see them.
struct DevGraph {
  const uint32_t *words;     // stream words (big-endian packing), >= 4 zero words of tail
  const uint64_t *offsets;   // n_c + 1 bit offsets by position
  const uint32_t *vertices;  // position -> vertex id (n)
  const uint32_t *deg;       // position -> degree (n)
  const uint32_t *small_off; // small CSR offsets by (position - n_c), n - n_c + 1
  const uint32_t *small_nbr; // small CSR neighbours
  uint64_t n;                // vertices
  uint64_t n_c;              // compressed vertices
};

// 64 stream bits starting at bit `pos`, MSB first.
template <class W>
__device__ __forceinline__ uint64_t win64(W w, uint64_t pos) {
  const uint64_t i = pos >> 5;
  const uint32_t s = uint32_t(pos) & 31u;
  const uint32_t a = w(i), b = w(i + 1), c = w(i + 2);
  const uint32_t hi = __funnelshift_l(b, a, s);
  const uint32_t lo = __funnelshift_l(c, b, s);
  return (uint64_t(hi) << 32) | lo;
}

// Global-memory word source (read-only path).
struct GWords {
  const uint32_t *__restrict__ p;
  GWords() = default;
  __device__ __forceinline__ GWords(const uint32_t *q) : p(q) {}
  __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return __ldg(p + i); }
};

// Words [lo, lo + n) from a shared-memory copy, every other word from global
// memory: a reader whose span was staged reads the copy, and anything outside
// the staged span (a clipped copy, a malformed stream) still reads the stream.
struct StagedWords {
  const uint32_t *__restrict__ g;  // the stream (global memory)
  const uint32_t *s;               // shared copy of words [lo, lo + n)
  uint64_t lo;
  uint32_t n;
  __device__ __forceinline__ uint32_t operator()(uint64_t i) const {
    const uint64_t k = i - lo;
    return k < n ? s[k] : __ldg(g + i);
  }
};

// Shared-memory word source: words [base_word, base_word + len) staged at s.
struct SWords {
  const uint32_t *s;
  uint64_t base_word;
  __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return s[i - base_word]; }
};

// gamma (graph_utils.cuh:63-67): z zeros, then the z+1 bits of x+1.
template <class W>
__device__ __forceinline__ uint32_t dec_gamma(W w, uint64_t &pos, bool &bad) {
  const uint64_t x = win64(w, pos);
  const uint32_t z = __clzll(x);
  if (z > 31) {
    bad = true;
    return 0;
  }
  pos += 2 * z + 1;
  return uint32_t(x >> (63 - 2 * z)) - 1u;
}

// zeta_3 (graph_utils.cuh:69-76): h zeros, a one, then 3(h+1) bits of x+1.
template <class W>
__device__ __forceinline__ uint32_t dec_zeta3(W w, uint64_t &pos, bool &bad) {
  const uint64_t x = win64(w, pos);
  const uint32_t h = __clzll(x);
  if (h > 10) {
    bad = true;
    return 0;
  }
  pos += 4 * (h + 1);
  return uint32_t((x << (h + 1)) >> (64 - 3 * (h + 1))) - 1u;
}

// decode_segment_cnt (graph_utils.cuh:88-97).
template <class W>
__device__ __forceinline__ uint32_t dec_segcnt(W w, uint64_t &pos, bool &bad) {
  const uint64_t x = win64(w, pos);
  const uint32_t z = __clzll(x);
  if (z == 0) {  // gamma(0): one segment, unless the next bit marks it empty
    if ((x >> 62) & 1ull) {
      pos += 2;
      return 0;
    }
    pos += 1;
    return 1;
  }
  if (z > 31) {
    bad = true;
    return 0;
  }
  pos += 2 * z + 1;
  return uint32_t(x >> (63 - 2 * z));  // gamma value + 1
}

// decode_first_num (graph_utils.cuh:34-37).
__device__ __forceinline__ uint32_t zigzag_first(uint32_t node, uint32_t x) {
  return (x & 1u) ? node - (x >> 1) - 1u : node + (x >> 1);
}

// Walks one vertex's neighbour list, calling emit(id) for every neighbour
// (intervals first, then residuals).  Returns the count, or -1 on a stream
// that leaves [pos, end), does not end at `end`, or names an id >= n.
template <class W, class Emit>
__device__ __forceinline__ int64_t walk_vertex(W w, uint64_t pos, uint64_t end, uint32_t node, uint64_t n,
                                               Emit emit) {
  bool bad = false;
  int64_t cnt_all = 0;
  // interval section (IntervalSegmentHelper, graph_utils.cuh:139-180)
  uint32_t nseg = dec_segcnt(w, pos, bad);
  const uint64_t ibase = pos;
  uint64_t last = pos;
  if (pos > end || nseg > (end - pos) / kSegBits + 1) return -1;
  for (uint32_t j = 0; j < nseg && !bad; j++) {
    uint64_t q = ibase + uint64_t(kSegBits) * j;
    if (q >= end) return -1;
    uint32_t cnt = dec_gamma(w, q, bad);
    uint32_t left = 0;
    for (uint32_t c = 0; c < cnt && !bad; c++) {
      uint32_t l = dec_gamma(w, q, bad);
      left = (c == 0) ? zigzag_first(node, l) : left + l + 1u;
      uint32_t len = dec_gamma(w, q, bad) + kMinItv;
      if (q > end || uint64_t(left) + len > n) return -1;
      for (uint32_t k = 0; k < len; k++) emit(left + k);
      cnt_all += len;
      left += len;
    }
    last = q;
  }
  pos = last;
  // residual section (ResidualSegmentHelper, graph_utils.cuh:100-137)
  nseg = dec_segcnt(w, pos, bad);
  const uint64_t rbase = pos;
  last = pos;
  if (pos > end || nseg > (end - pos) / kSegBits + 1) return -1;
  for (uint32_t j = 0; j < nseg && !bad; j++) {
    uint64_t q = rbase + uint64_t(kSegBits) * j;
    if (q >= end) return -1;
    uint32_t cnt = dec_gamma(w, q, bad);
    uint32_t v = 0;
    for (uint32_t c = 0; c < cnt && !bad; c++) {
      uint32_t x = dec_zeta3(w, q, bad);
      v = (c == 0) ? zigzag_first(node, x) : v + x + 1u;
      if (q > end || uint64_t(v) >= n) return -1;
      emit(v);
      cnt_all++;
    }
    last = q;
  }
  if (bad || last != end) return -1;
  return cnt_all;
}

// Sequential MSB-first reader with a 64-bit register buffer: one 32-bit load
// per 32 bits consumed.  Codes that do not fit the buffer's fast path (gamma
// with >= 16 leading zeros, zeta with >= 8) are read through win64.
// ---------------------------------------------------------- bulk copies ---
// 1-D bulk copies global -> shared memory by the copy engine
// (cp.async.bulk, sm_90+), completed on an mbarrier in shared memory.  Never
// with cluster multicast.  Source and destination 16-byte aligned, size a
// multiple of 16.
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return uint32_t(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
// makes initialised mbarriers visible to the copy engine
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// orders this thread's earlier generic accesses to shared memory before
// later bulk-copy writes to it
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// one arrival that also expects `bytes` of copies to complete on bar, then
// the copy itself
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0u;
}
// Waits for phase `parity` of bar to complete, giving up after `limit` tries
// (each try suspends the thread for a bounded time).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; i++)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}

// WS: the word source (GWords, or StagedWords for a span staged in shared
// memory).
template <class WS>
struct BitReaderT {
  // a global-memory source is read through a pointer to the next word (a
  // refill is one load and one pointer step, no index arithmetic)
  static constexpr bool kPtr = std::is_same<WS, GWords>::value;
  WS w;
  uint32_t hi, lo;       // upcoming bits, MSB-aligned: hi the next 32, lo the 32 after (zero past the valid bits)
  uint64_t wnext;        // next word to load (sources other than GWords)
  const uint32_t *wp;    // GWords: the next word to load
  uint32_t nb;           // valid bits in hi:lo

  __device__ __forceinline__ uint64_t next_word() const {
    if constexpr (kPtr) return uint64_t(wp - w.p);
    else return wnext;
  }
  // absolute position of the next unread bit (kept implicit: every code
  // would otherwise pay a 64-bit add)
  __device__ __forceinline__ uint64_t pos() const { return (next_word() << 5) - nb; }
  __device__ __forceinline__ void seek(WS words, uint64_t p) {
    w = words;
    const uint64_t i = p >> 5;
    const uint32_t s = uint32_t(p) & 31u;
    const uint32_t a = w(i), b = w(i + 1);
    hi = __funnelshift_l(b, a, s);
    lo = b << s;
    nb = 64 - s;
    if constexpr (kPtr) wp = w.p + i + 2;
    else wnext = i + 2;
  }
  // Tops the buffer up to at least 33 valid bits (from at least 1).
  __device__ __forceinline__ void fill() {
    if (nb <= 32) {  // every valid bit is in hi and lo is zero
      uint32_t x;
      if constexpr (kPtr) x = __ldg(wp++);
      else x = w(wnext++);
      hi |= __funnelshift_rc(x, 0u, nb);  // x >> nb, 0 when nb == 32
      lo = x << (32 - nb);
      nb += 32;
    }
  }
  __device__ __forceinline__ void skip(uint32_t k) {  // k <= 32, k <= nb
    hi = __funnelshift_lc(lo, hi, k);
    lo = __funnelshift_lc(0u, lo, k);  // lo << k, 0 when k == 32
    nb -= k;
  }
  // After fill() hi is all valid bits (nb >= 33); a fast-path code lies
  // within it, so its fields come from 32-bit shifts.
  __device__ __forceinline__ uint32_t gamma(bool &bad) {
    fill();
    const uint32_t z = __clz(hi);
    if (z < 16) {  // 2z+1 <= 31 bits
      const uint32_t len = 2 * z + 1;
      const uint32_t v = hi >> (32 - len);
      skip(len);
      return v - 1u;
    }
    uint64_t p = pos();
    const uint32_t v = dec_gamma(w, p, bad);
    seek(w, p);
    return v;
  }
  __device__ __forceinline__ uint32_t zeta3(bool &bad) {
    fill();
    const uint32_t h = __clz(hi);
    if (h < 8) {  // 4(h+1) <= 32 bits
      const uint32_t v = (hi << (h + 1)) >> (32 - 3 * (h + 1));
      skip(4 * (h + 1));
      return v - 1u;
    }
    uint64_t p = pos();
    const uint32_t v = dec_zeta3(w, p, bad);
    seek(w, p);
    return v;
  }
  __device__ __forceinline__ uint32_t segcnt(bool &bad) {
    fill();
    if (hi >> 31) {
      if ((hi >> 30) & 1u) {
        skip(2);
        return 0;
      }
      skip(1);
      return 1;
    }
    return gamma(bad) + 1u;
  }
};
using BitReader = BitReaderT<GWords>;

// Walks one vertex with the buffered reader (same contract as walk_vertex).
// kOncePerSegment: a residual segment's ids are emitted clamped to n - 1 and
// its end and largest (last) id are tested once, after its last code, instead
// of after every code; the result is the same for a stream the code-by-code
// form (the validation at create) accepted.  In a loop whose lanes diverge,
// every test is paid by the whole warp (k_packed on the road grid 1404^2:
// 0.118 -> 0.070 ms per iteration).
template <bool kOncePerSegment = false, class Emit>
__device__ __forceinline__ int64_t walk_vertex_buf(const uint32_t *__restrict__ words, uint64_t pos, uint64_t end,
                                                   uint32_t node, uint64_t n, Emit emit,
                                                   int64_t *interval_items = nullptr) {
  bool bad = false;
  int64_t cnt_all = 0;
  BitReader r;
  r.seek(words, pos);
  uint32_t nseg = r.segcnt(bad);
  const uint64_t ibase = r.pos();
  uint64_t last = r.pos();
  if (bad || r.pos() > end || nseg > (end - r.pos()) / kSegBits + 1) return -1;
  for (uint32_t j = 0; j < nseg; j++) {
    const uint64_t q = ibase + uint64_t(kSegBits) * j;
    if (q >= end) return -1;
    if (j) r.seek(words, q);
    const uint32_t cnt = r.gamma(bad);
    uint32_t left = 0;
    for (uint32_t c = 0; c < cnt; c++) {
      const uint32_t l = r.gamma(bad);
      left = (c == 0) ? zigzag_first(node, l) : left + l + 1u;
      const uint32_t len = r.gamma(bad) + kMinItv;
      if (bad || r.pos() > end || uint64_t(left) + len > n) return -1;
      for (uint32_t k = 0; k < len; k++) emit(left + k);
      cnt_all += len;
      left += len;
    }
    last = r.pos();
  }
  if (interval_items) *interval_items = cnt_all;
  // the reader already stands at `last`: the residual section follows the last
  // interval segment's final item (or the empty interval section)
  nseg = r.segcnt(bad);
  const uint64_t rbase = r.pos();
  last = r.pos();
  if (bad || r.pos() > end || nseg > (end - r.pos()) / kSegBits + 1) return -1;
  for (uint32_t j = 0; j < nseg; j++) {
    const uint64_t q = rbase + uint64_t(kSegBits) * j;
    if (q >= end) return -1;
    if (j) r.seek(words, q);
    const uint32_t cnt = r.gamma(bad);
    uint32_t v = 0;
    if constexpr (kOncePerSegment) {
      const uint32_t nmax = uint32_t(n - 1);
      if (cnt) {
        v = zigzag_first(node, r.zeta3(bad));
        emit(min(v, nmax));
      }
      for (uint32_t c = 1; c < cnt; c++) {
        v += r.zeta3(bad) + 1u;
        emit(min(v, nmax));
      }
      if (cnt && (bad || r.pos() > end || v > nmax)) return -1;
      cnt_all += cnt;
    } else {
      for (uint32_t c = 0; c < cnt; c++) {
        const uint32_t x = r.zeta3(bad);
        v = (c == 0) ? zigzag_first(node, x) : v + x + 1u;
        if (bad || r.pos() > end || uint64_t(v) >= n) return -1;
        emit(v);
        cnt_all++;
      }
    }
    last = r.pos();
  }
  if (bad || last != end) return -1;
  return cnt_all;
}

// ---------------------------------------------------------------- hashing --
// Count-min-sketch row hashes, include/cms.cuh:96-132 (cm_hash1..cm_hash4).
__device__ __forceinline__ uint32_t cm_hash(int r, uint32_t k) {
  switch (r) {
    case 0:
      k ^= k >> 16; k *= 0x12ebcb3bu; k ^= k >> 13; k *= 0xc123ae53u; k ^= k >> 16;
      return k;
    case 1:
      k ^= k >> 16; k *= 0x21eb21bbu; k ^= k >> 13; k *= 0x2cb2ea35u; k ^= k >> 16;
      return k;
    case 2:
      k ^= k >> 16; k *= 0x8febce61u; k ^= k >> 13; k *= 0xa2b2be25u; k ^= k >> 16;
      return k;
    default:
      k ^= k >> 12; k *= 0x13ebdb3au; k ^= k >> 12; k *= 0xc123ae53u; k ^= k >> 14;
      return k;
  }
}

// Slot hash for the exact-count tables (a murmur3-style finaliser).
__device__ __forceinline__ uint32_t slot_hash(uint32_t k) {
  k ^= k >> 16;
  k *= 0x7feb352du;
  k ^= k >> 15;
  k *= 0x846ca68bu;
  k ^= k >> 16;
  return k;
}

// (count, label) packed so that a larger value means a better label: more
// occurrences first, then the smaller label.
__device__ __forceinline__ uint64_t pack_best(uint32_t count, uint32_t label) {
  return (uint64_t(count) << 32) | uint64_t(~label);
}
__device__ __forceinline__ uint32_t best_label(uint64_t packed) { return ~uint32_t(packed); }

// The warp's largest 64-bit value: the largest high word, then the largest
// low word among the lanes that hold it (two redux instructions instead of
// five 64-bit shuffle rounds: count pass 2.32 -> 2.26 ms at R-MAT scale 24).
// Called by all 32 lanes.
__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v) {
  const uint32_t hi = __reduce_max_sync(kFull, uint32_t(v >> 32));
  const uint32_t lo = __reduce_max_sync(kFull, uint32_t(v >> 32) == hi ? uint32_t(v) : 0u);
  return (uint64_t(hi) << 32) | lo;
}

// Open-addressing exact counter in shared (or global) memory.  Keys are
// stored as label + 1 so that 0 marks an empty slot.  cap is a power of two
// larger than the number of distinct labels inserted.
__device__ __forceinline__ void table_add(uint32_t *keys, uint32_t *cnts, uint32_t cap, uint32_t label,
                                          uint32_t c) {
  const uint32_t key = label + 1u;
  uint32_t h = slot_hash(label) & (cap - 1);
  for (uint32_t probe = 0; probe < cap; probe++) {
    uint32_t k = keys[h];
    if (k == key) {
      atomicAdd(&cnts[h], c);
      return;
    }
    if (k == 0) {
      uint32_t old = atomicCAS(&keys[h], 0u, key);
      if (old == 0u || old == key) {
        atomicAdd(&cnts[h], c);
        return;
      }
    }
    h = (h + 1) & (cap - 1);
  }
}

// Exact counter in shared memory without clearing: a slot is one 64-bit word
// [epoch:16 | label:32 | count:16].  A slot whose epoch is not the current
// one is empty, so a new vertex only bumps the epoch.  insert() returns the
// label's count after the increment, so the caller keeps a running argmax and
// never scans the table.  cap (a power of two) must exceed the number of
// distinct labels inserted under one epoch; counts must stay below 65536.
struct EpochTable {
  unsigned long long *slots;
  uint32_t cap;
  uint32_t epoch;  // 1..65535
  // Triangular probing (h, h+1, h+3, h+6, ...) visits every slot of a
  // power-of-two table and keeps probe chains short at high load.
  __device__ __forceinline__ uint32_t insert(uint32_t label, uint32_t c) const {
    const unsigned long long tag = (uint64_t(epoch) << 48) | (uint64_t(label) << 16);
    uint32_t h = slot_hash(label) & (cap - 1), step = 0;
    for (uint32_t probe = 0; probe < 2 * cap; probe++) {
      const unsigned long long v = slots[h];
      if (uint32_t(v >> 48) == epoch) {
        if ((v & ~0xFFFFull) == tag) {
          const unsigned long long old = atomicAdd(&slots[h], (unsigned long long)c);
          return uint32_t(old & 0xFFFFull) + c;
        }
        h = (h + ++step) & (cap - 1);
        continue;
      }
      if (atomicCAS(&slots[h], v, tag | c) == v) return c;
      // another lane claimed the slot first: look at it again
    }
    return 0;
  }
};

// Folds lanes holding equal labels into one lane: returns the number of lanes
// folded into this one (the lowest lane of each label; 0 for the others, or
// when !ok).  One match.any finds every lane's equals at once; measured
// against folding by ballot rounds (up to four shuffle + ballot rounds) it
// took the R-MAT scale-24 count pass from 2.40 to 2.34 ms.  Called by all 32
// lanes.
__device__ __forceinline__ uint32_t warp_merge(bool ok, uint32_t lab) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t okm = __ballot_sync(0xFFFFFFFFu, ok);
  const uint32_t m = __match_any_sync(0xFFFFFFFFu, lab) & okm;
  if (!ok) return 0u;
  return (uint32_t(__ffs(m) - 1) == lane) ? uint32_t(__popc(m)) : 0u;
}

// For every lane, how many lanes of its group (gm: the group's lane mask, gl:
// the group index, groups of a power-of-two size) hold its label; 0 when !ok.
// Two ballot rounds settle the groups' most common labels; lanes left after
// them are counted with match.any.  Called by all 32 lanes.
__device__ __forceinline__ uint32_t group_counts(bool ok, uint32_t lab, uint32_t gm, uint32_t gl) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t rest = __ballot_sync(0xFFFFFFFFu, ok);
  uint32_t cnt = 0;
  for (int r = 0; r < 2 && rest; r++) {
    const uint32_t mine = rest & gm;
    const uint32_t ld = mine ? uint32_t(__ffs(mine) - 1) : lane;
    const uint32_t x = __shfl_sync(0xFFFFFFFFu, lab, ld);
    const bool hit = ((mine >> lane) & 1u) && lab == x;
    const uint32_t hits = __ballot_sync(0xFFFFFFFFu, hit);
    if (hit) cnt = uint32_t(__popc(hits & gm));
    rest &= ~hits;
  }
  if (rest) {
    const bool rem = (rest >> lane) & 1u;
    const unsigned long long key = rem ? ((uint64_t(gl) << 32) | lab) : (0xFFFFFFFF00000000ull | lane);
    const uint32_t m = __match_any_sync(0xFFFFFFFFu, key);
    if (rem) cnt = uint32_t(__popc(m));
  }
  return cnt;
}

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// The GPU's nanosecond clock (the same for every SM).
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bulk prefetch of [p, p + bytes) into L2 (cp.async.bulk.prefetch, sm_90+):
// one instruction per range, rounded out to 16-byte boundaries, split into
// pieces below 1 MiB.
__device__ __forceinline__ void prefetch_l2(const void *p, uint64_t bytes) {
  if (!p || bytes == 0) return;
  uint64_t a = reinterpret_cast<uint64_t>(p) & ~uint64_t(15);
  const uint64_t e = (reinterpret_cast<uint64_t>(p) + bytes + 15) & ~uint64_t(15);
  while (a < e) {
    const uint32_t n = uint32_t(e - a < (1u << 20) ? e - a : (1u << 20));
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(n) : "memory");
    a += n;
  }
}

}  // namespace lpa_dev
