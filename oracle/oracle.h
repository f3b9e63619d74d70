/*
 * CPU oracle for synchronous label propagation over a CGR-compressed graph.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the GPU path is compared
 * against; the product (lpa_b200) never links, loads or calls it.  It is a
 * plain-C restatement of the reference algorithm:
 *   - CGR bit reader and segment decode: include/graph_utils.cuh:19-180
 *     (CgrReader, ResidualSegmentHelper, IntervalSegmentHelper), widened to
 *     64-bit bit positions (the reference reader uses uint32 positions,
 *     include/graph_utils.cuh:13,22, which overflow past 2^32 bits);
 *   - section/segment layout: src/compressor.cpp:330-515 (intervalize,
 *     encode_intervals, encode_residuals, append_segment);
 *   - word packing of the .graph file: src/file.cpp:216-239 (big-endian
 *     32-bit words, bit i = bit 31-(i%32) of word i/32);
 *   - count-min-sketch row hashes: include/cms.cuh:96-132 (cm_hash1..4);
 *   - the update rule of one synchronous iteration (most frequent neighbour
 *     label, smallest label wins ties; count-min sketch of depth 4 and width
 *     1024 at or above the sketch threshold; isolated vertices keep their
 *     label; double-buffered labels).
 */
#ifndef LPA_ORACLE_H
#define LPA_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_CMS_DEPTH 4
#define ORC_CMS_WIDTH 1024

/* Decode the neighbour list of one compressed vertex whose bits are
 * [bit_begin, bit_end) of the stream.  Neighbours are written in stream order
 * (intervals first, then residuals) into out[0..cap).  Returns the number of
 * neighbours, or -1 on a malformed stream (decode overran bit_end, did not end
 * exactly at bit_end), or -2 when more than cap neighbours. */
int64_t orc_decode_vertex(const uint32_t *words, uint64_t nwords,
                          uint64_t bit_begin, uint64_t bit_end, uint32_t node,
                          uint32_t *out, uint64_t cap);

/* Number of neighbours of one compressed vertex (same checks as above). */
int64_t orc_vertex_degree(const uint32_t *words, uint64_t nwords,
                          uint64_t bit_begin, uint64_t bit_end, uint32_t node);

/* Decode the whole mixed graph (CGR part + small CSR part) into a CSR indexed
 * by vertex id, with each list sorted ascending (the order of the reference's
 * .clm).  row_out has n+1 entries; clm_out must hold m entries, where m is
 * obtained from a first call with clm_out == NULL (returns m).  Returns the
 * number of arcs, or -1 on a malformed stream. */
int64_t orc_decode_csr(const uint32_t *words, uint64_t nwords,
                       const uint64_t *offsets, uint64_t n_c,
                       const uint32_t *vertices, uint64_t n,
                       const uint32_t *small_graph, const uint32_t *small_offset,
                       uint64_t *row_out, uint32_t *clm_out);

/* Row hash of the count-min sketch: cm_hash_{r+1}(key ^ seed_r) % width. */
uint32_t orc_cms_index(int r, uint32_t key, uint32_t seed_r);

/* The per-row seeds derived from one 64-bit sketch seed. */
void orc_cms_seeds(uint64_t cms_seed, uint32_t seeds_out[ORC_CMS_DEPTH]);

/* One synchronous iteration on a CSR: lab_out[v] from lab_in.  Vertices with
 * degree >= cms_thr (cms_thr != 0) use the sketch.  Returns the changed count. */
uint64_t orc_lp_iterate_csr(const uint64_t *row, const uint32_t *clm, uint64_t n,
                            const uint32_t *lab_in, uint32_t *lab_out,
                            uint64_t cms_thr, uint64_t cms_seed, int threads);

/* One synchronous iteration straight from the compressed form (decode each
 * vertex, gather, count) -- the CPU path timed as the baseline.  Returns the
 * changed count, or UINT64_MAX on a malformed stream. */
uint64_t orc_lp_iterate_cgr(const uint32_t *words, uint64_t nwords,
                            const uint64_t *offsets, uint64_t n_c,
                            const uint32_t *vertices, uint64_t n,
                            const uint32_t *small_graph, const uint32_t *small_offset,
                            const uint32_t *lab_in, uint32_t *lab_out,
                            uint64_t cms_thr, uint64_t cms_seed, int threads,
                            uint64_t pos_begin, uint64_t pos_end);

/* Arcs of positions [pos_begin, pos_end) (UINT64_MAX on a malformed stream). */
uint64_t orc_range_arcs(const uint32_t *words, uint64_t nwords, const uint64_t *offsets, uint64_t n_c,
                        const uint32_t *vertices, const uint32_t *small_offset, uint64_t pos_begin,
                        uint64_t pos_end);

#ifdef __cplusplus
}
#endif
#endif
