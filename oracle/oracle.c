/*
 * CPU oracle: restatement of the reference's CGR decode and of one synchronous
 * label-propagation iteration.  TEST INFRASTRUCTURE ONLY -- see oracle.h for
 * the reference files each part follows.  Nothing in the product links this.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Bit reader (include/graph_utils.cuh:19-98, CgrReader), 64-bit positions.  */
/* ------------------------------------------------------------------------ */
typedef struct {
  const uint32_t *w;
  uint64_t nw;
  uint64_t pos;
  int bad;
} rd_t;

static inline uint32_t word_at(const rd_t *r, uint64_t i) {
  return i < r->nw ? r->w[i] : 0u;
}

/* 64 stream bits starting at the cursor, MSB first (CgrReader::cur widened). */
static inline uint64_t win64(const rd_t *r) {
  uint64_t i = r->pos >> 5;
  unsigned s = (unsigned)(r->pos & 31u);
  uint64_t hi = ((uint64_t)word_at(r, i) << 32) | word_at(r, i + 1);
  if (s == 0) return hi;
  return (hi << s) | ((uint64_t)word_at(r, i + 2) >> (32 - s));
}

/* decode_unary (graph_utils.cuh:48-54): skips the zeros, returns zeros + 1. */
static inline uint32_t rd_unary(rd_t *r) {
  uint64_t w = win64(r);
  if (w == 0) { r->bad = 1; return 1; }
  uint32_t z = (uint32_t)__builtin_clzll(w);
  if (z > 31) { r->bad = 1; return 1; }
  r->pos += z;
  return z + 1;
}

/* decode_int (graph_utils.cuh:56-61): the next len bits as an integer. */
static inline uint64_t rd_int(rd_t *r, uint32_t len) {
  uint64_t x = win64(r) >> (64 - len);
  r->pos += len;
  return x;
}

/* decode_gamma (graph_utils.cuh:63-67). */
static inline uint32_t rd_gamma(rd_t *r) {
  uint32_t h = rd_unary(r);
  return (uint32_t)(rd_int(r, h) - 1);
}

/* decode_zeta with k = 3 (graph_utils.cuh:69-76). */
static inline uint32_t rd_zeta(rd_t *r) {
  uint32_t h = rd_unary(r);
  r->pos += 1;
  return (uint32_t)(rd_int(r, h * 3) - 1);
}

/* decode_segment_cnt (graph_utils.cuh:88-97): a section holding one empty
 * segment is written as gamma(0) gamma(0) = "11" and reads as zero segments. */
static inline uint32_t rd_segment_cnt(rd_t *r) {
  uint32_t cnt = rd_gamma(r) + 1;
  if (cnt == 1 && (win64(r) >> 63)) {
    r->pos += 1;
    cnt = 0;
  }
  return cnt;
}

/* decode_first_num (graph_utils.cuh:34-37): zig-zag value relative to node. */
static inline uint32_t first_num(uint32_t node, uint32_t x) {
  return (x & 1u) ? node - (x >> 1) - 1u : node + (x >> 1);
}

#define SEG_BITS 256u /* INTERVAL_SEGMENT_LEN, graph_utils.cuh:17; src/file.cpp:84 */
#define MIN_ITV 4u    /* min interval length, graph_utils.cuh:172; src/file.cpp:84 */

/* Walks one vertex.  When out != NULL writes neighbours (up to cap).  Returns
 * the neighbour count, -1 on a malformed stream, -2 when out overflows cap.
 * Layout: src/compressor.cpp:364-515. */
static int64_t walk_vertex(const uint32_t *words, uint64_t nwords, uint64_t bit_begin,
                           uint64_t bit_end, uint32_t node, uint32_t *out, uint64_t cap) {
  rd_t r = {words, nwords, bit_begin, 0};
  uint64_t n = 0;

  /* interval section: IntervalSegmentHelper (graph_utils.cuh:139-180) */
  uint32_t nseg = rd_segment_cnt(&r);
  uint64_t base = r.pos, end = r.pos;
  for (uint32_t j = 0; j < nseg && !r.bad; j++) {
    r.pos = base + (uint64_t)SEG_BITS * j;
    if (r.pos >= bit_end) return -1;
    uint32_t cnt = rd_gamma(&r);
    uint32_t left = 0;
    for (uint32_t c = 0; c < cnt && !r.bad; c++) {
      if (c == 0) left = first_num(node, rd_gamma(&r));
      else left += rd_gamma(&r) + 1u;
      uint32_t len = rd_gamma(&r) + MIN_ITV;
      if (r.pos > bit_end) return -1;
      if (out) {
        if (n + len > cap) return -2;
        for (uint32_t k = 0; k < len; k++) out[n + k] = left + k;
      }
      n += len;
      left += len;
    }
    /* every segment but the last is padded to SEG_BITS */
    if (j + 1 < nseg && r.pos > base + (uint64_t)SEG_BITS * (j + 1)) return -1;
    end = r.pos;
  }
  r.pos = end;

  /* residual section: ResidualSegmentHelper (graph_utils.cuh:100-137) */
  nseg = rd_segment_cnt(&r);
  base = r.pos;
  end = r.pos;
  for (uint32_t j = 0; j < nseg && !r.bad; j++) {
    r.pos = base + (uint64_t)SEG_BITS * j;
    if (r.pos >= bit_end) return -1;
    uint32_t cnt = rd_gamma(&r);
    uint32_t v = 0;
    for (uint32_t c = 0; c < cnt && !r.bad; c++) {
      if (c == 0) v = first_num(node, rd_zeta(&r));
      else v += rd_zeta(&r) + 1u;
      if (r.pos > bit_end) return -1;
      if (out) {
        if (n >= cap) return -2;
        out[n] = v;
      }
      n++;
    }
    if (j + 1 < nseg && r.pos > base + (uint64_t)SEG_BITS * (j + 1)) return -1;
    end = r.pos;
  }
  if (r.bad || end != bit_end) return -1;
  return (int64_t)n;
}

int64_t orc_decode_vertex(const uint32_t *words, uint64_t nwords, uint64_t bit_begin,
                          uint64_t bit_end, uint32_t node, uint32_t *out, uint64_t cap) {
  return walk_vertex(words, nwords, bit_begin, bit_end, node, out, cap);
}

int64_t orc_vertex_degree(const uint32_t *words, uint64_t nwords, uint64_t bit_begin,
                          uint64_t bit_end, uint32_t node) {
  return walk_vertex(words, nwords, bit_begin, bit_end, node, NULL, 0);
}

/* ------------------------------------------------------------------------ */
/* Sorting helpers                                                           */
/* ------------------------------------------------------------------------ */
static void sort_u32(uint32_t *a, uint64_t n, uint32_t *tmp) {
  if (n <= 48) {
    for (uint64_t i = 1; i < n; i++) {
      uint32_t x = a[i];
      uint64_t j = i;
      while (j > 0 && a[j - 1] > x) { a[j] = a[j - 1]; j--; }
      a[j] = x;
    }
    return;
  }
  /* LSD radix, 4 passes of 8 bits */
  uint32_t *src = a, *dst = tmp;
  for (int sh = 0; sh < 32; sh += 8) {
    uint64_t cnt[257];
    memset(cnt, 0, sizeof(cnt));
    for (uint64_t i = 0; i < n; i++) cnt[((src[i] >> sh) & 255u) + 1]++;
    for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
    for (uint64_t i = 0; i < n; i++) dst[cnt[(src[i] >> sh) & 255u]++] = src[i];
    uint32_t *t = src; src = dst; dst = t;
  }
  /* 4 passes: result is back in a */
}

/* ------------------------------------------------------------------------ */
/* CSR decode                                                                */
/* ------------------------------------------------------------------------ */
int64_t orc_decode_csr(const uint32_t *words, uint64_t nwords, const uint64_t *offsets,
                       uint64_t n_c, const uint32_t *vertices, uint64_t n,
                       const uint32_t *small_graph, const uint32_t *small_offset,
                       uint64_t *row_out, uint32_t *clm_out) {
  uint64_t *deg = (uint64_t *)calloc(n + 1, sizeof(uint64_t));
  if (!deg) return -1;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 256)
  for (uint64_t p = 0; p < n; p++) {
    uint32_t v = vertices[p];
    if (v >= n) { bad = 1; continue; }
    int64_t d;
    if (p < n_c) d = orc_vertex_degree(words, nwords, offsets[p], offsets[p + 1], v);
    else d = (int64_t)small_offset[p - n_c + 1] - (int64_t)small_offset[p - n_c];
    if (d < 0) bad = 1;
    else deg[v] = (uint64_t)d;
  }
  if (bad) { free(deg); return -1; }
  uint64_t m = 0;
  for (uint64_t v = 0; v < n; v++) {
    if (row_out) row_out[v] = m;
    m += deg[v];
  }
  if (row_out) row_out[n] = m;
  if (clm_out && row_out) {
#pragma omp parallel
    {
      uint64_t tcap = 0;
      uint32_t *tmp = NULL;
#pragma omp for schedule(dynamic, 256)
      for (uint64_t p = 0; p < n; p++) {
        uint32_t v = vertices[p];
        uint32_t *dst = clm_out + row_out[v];
        uint64_t d = deg[v];
        if (p < n_c) {
          if (walk_vertex(words, nwords, offsets[p], offsets[p + 1], v, dst, d) != (int64_t)d) bad = 1;
        } else {
          memcpy(dst, small_graph + small_offset[p - n_c], d * sizeof(uint32_t));
        }
        if (d > tcap) {
          free(tmp);
          tcap = d;
          tmp = (uint32_t *)malloc(tcap * sizeof(uint32_t));
        }
        sort_u32(dst, d, tmp);
      }
      free(tmp);
    }
  }
  free(deg);
  return bad ? -1 : (int64_t)m;
}

/* ------------------------------------------------------------------------ */
/* Count-min sketch row hashes (include/cms.cuh:96-132, cm_hash1..cm_hash4)   */
/* ------------------------------------------------------------------------ */
static inline uint32_t cm_hash(int r, uint32_t k) {
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

uint32_t orc_cms_index(int r, uint32_t key, uint32_t seed_r) {
  return cm_hash(r, key ^ seed_r) % ORC_CMS_WIDTH;
}

/* seed_r = low32(seed) XOR (0x9E3779B9 * (r + 1)), high32(seed) folded in. */
void orc_cms_seeds(uint64_t cms_seed, uint32_t seeds_out[ORC_CMS_DEPTH]) {
  uint32_t lo = (uint32_t)cms_seed, hi = (uint32_t)(cms_seed >> 32);
  for (int r = 0; r < ORC_CMS_DEPTH; r++)
    seeds_out[r] = (lo ^ (0x9E3779B9u * (uint32_t)(r + 1))) + hi * 0x85EBCA6Bu;
}

/* ------------------------------------------------------------------------ */
/* The update rule for one vertex                                            */
/* ------------------------------------------------------------------------ */
typedef struct {
  uint32_t *a, *b;
  uint64_t cap;
  uint32_t cms[ORC_CMS_DEPTH * ORC_CMS_WIDTH];
} scratch_t;

static void scratch_reserve(scratch_t *s, uint64_t d) {
  if (d <= s->cap) return;
  free(s->a);
  free(s->b);
  s->cap = d < 1024 ? 1024 : d;
  s->a = (uint32_t *)malloc(s->cap * sizeof(uint32_t));
  s->b = (uint32_t *)malloc(s->cap * sizeof(uint32_t));
}

/* labs[0..d) holds the neighbour labels (clobbered).  Exact: most frequent,
 * ties to the smallest.  Sketch: argmax of min_r C[r][h_r(l)] over distinct
 * neighbour labels, ties to the smallest. */
static uint32_t pick_label(uint32_t *labs, uint64_t d, scratch_t *s, uint64_t cms_thr,
                           const uint32_t seeds[ORC_CMS_DEPTH]) {
  if (cms_thr != 0 && d >= cms_thr) {
    memset(s->cms, 0, sizeof(s->cms));
    for (uint64_t i = 0; i < d; i++)
      for (int r = 0; r < ORC_CMS_DEPTH; r++)
        s->cms[r * ORC_CMS_WIDTH + orc_cms_index(r, labs[i], seeds[r])]++;
    uint32_t best = 0, best_est = 0;
    int have = 0;
    for (uint64_t i = 0; i < d; i++) {
      uint32_t l = labs[i], est = UINT32_MAX;
      for (int r = 0; r < ORC_CMS_DEPTH; r++) {
        uint32_t c = s->cms[r * ORC_CMS_WIDTH + orc_cms_index(r, l, seeds[r])];
        if (c < est) est = c;
      }
      if (!have || est > best_est || (est == best_est && l < best)) {
        best = l;
        best_est = est;
        have = 1;
      }
    }
    return best;
  }
  sort_u32(labs, d, s->b);
  uint32_t best = labs[0];
  uint64_t best_cnt = 0, i = 0;
  while (i < d) {
    uint64_t j = i + 1;
    while (j < d && labs[j] == labs[i]) j++;
    if (j - i > best_cnt) { /* strictly greater: the first (smallest) wins ties */
      best_cnt = j - i;
      best = labs[i];
    }
    i = j;
  }
  return best;
}

uint64_t orc_lp_iterate_csr(const uint64_t *row, const uint32_t *clm, uint64_t n,
                            const uint32_t *lab_in, uint32_t *lab_out, uint64_t cms_thr,
                            uint64_t cms_seed, int threads) {
  uint32_t seeds[ORC_CMS_DEPTH];
  orc_cms_seeds(cms_seed, seeds);
  uint64_t changed = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel reduction(+ : changed)
  {
    scratch_t *s = (scratch_t *)calloc(1, sizeof(scratch_t));
#pragma omp for schedule(dynamic, 1024)
    for (uint64_t v = 0; v < n; v++) {
      uint64_t d = row[v + 1] - row[v];
      uint32_t nl = lab_in[v];
      if (d > 0) {
        scratch_reserve(s, d);
        for (uint64_t i = 0; i < d; i++) s->a[i] = lab_in[clm[row[v] + i]];
        nl = pick_label(s->a, d, s, cms_thr, seeds);
      }
      lab_out[v] = nl;
      changed += (nl != lab_in[v]);
    }
    free(s->a);
    free(s->b);
    free(s);
  }
  return changed;
}

uint64_t orc_lp_iterate_cgr(const uint32_t *words, uint64_t nwords, const uint64_t *offsets,
                            uint64_t n_c, const uint32_t *vertices, uint64_t n,
                            const uint32_t *small_graph, const uint32_t *small_offset,
                            const uint32_t *lab_in, uint32_t *lab_out, uint64_t cms_thr,
                            uint64_t cms_seed, int threads, uint64_t pos_begin,
                            uint64_t pos_end) {
  uint32_t seeds[ORC_CMS_DEPTH];
  orc_cms_seeds(cms_seed, seeds);
  if (pos_end > n) pos_end = n;
  uint64_t changed = 0;
  int bad = 0;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
#pragma omp parallel reduction(+ : changed)
  {
    scratch_t *s = (scratch_t *)calloc(1, sizeof(scratch_t));
    uint64_t ids_cap = 4096;
    uint32_t *ids = (uint32_t *)malloc(ids_cap * sizeof(uint32_t));
#pragma omp for schedule(dynamic, 1024)
    for (uint64_t p = pos_begin; p < pos_end; p++) {
      uint32_t v = vertices[p];
      int64_t d;
      const uint32_t *nb;
      if (p < n_c) {
        for (;;) {
          d = walk_vertex(words, nwords, offsets[p], offsets[p + 1], v, ids, ids_cap);
          if (d != -2) break;
          free(ids);
          ids_cap *= 2;
          ids = (uint32_t *)malloc(ids_cap * sizeof(uint32_t));
        }
        if (d < 0) { bad = 1; continue; }
        nb = ids;
      } else {
        d = (int64_t)small_offset[p - n_c + 1] - (int64_t)small_offset[p - n_c];
        nb = small_graph + small_offset[p - n_c];
      }
      uint32_t nl = lab_in[v];
      if (d > 0) {
        scratch_reserve(s, (uint64_t)d);
        for (int64_t i = 0; i < d; i++) s->a[i] = lab_in[nb[i]];
        nl = pick_label(s->a, (uint64_t)d, s, cms_thr, seeds);
      }
      lab_out[v] = nl;
      changed += (nl != lab_in[v]);
    }
    free(ids);
    free(s->a);
    free(s->b);
    free(s);
  }
  return bad ? UINT64_MAX : changed;
}

uint64_t orc_range_arcs(const uint32_t *words, uint64_t nwords, const uint64_t *offsets, uint64_t n_c,
                        const uint32_t *vertices, const uint32_t *small_offset, uint64_t pos_begin,
                        uint64_t pos_end) {
  uint64_t arcs = 0;
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : arcs)
  for (uint64_t p = pos_begin; p < pos_end; p++) {
    if (p < n_c) {
      int64_t d = orc_vertex_degree(words, nwords, offsets[p], offsets[p + 1], vertices[p]);
      if (d < 0) bad = 1;
      else arcs += (uint64_t)d;
    } else {
      arcs += small_offset[p - n_c + 1] - small_offset[p - n_c];
    }
  }
  return bad ? UINT64_MAX : arcs;
}
