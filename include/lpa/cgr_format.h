// CGR (compressed graph representation) format layer: in-memory containers and
// the fast parallel encoder.
//
// The bit layout is the reference's (src/compressor.cpp:306-515, written by
// write_bit_array src/compressor.cpp:178-290 and read back by
// File::load_compress_graph src/file.cpp:197-262):
//   * per vertex: an interval section then a residual section;
//   * a section is gamma(#segments - 1) followed by the segments; every
//     segment but the last is zero-padded to `seg_len` bits; a segment is
//     gamma(#items) followed by the items; the first item of each segment is
//     zig-zag coded relative to the vertex id, the others as gaps;
//   * interval item = gamma(left) gamma(len - min_itv_len); residual item =
//     zeta_k(value);
//   * vertices are ordered large (deg >= large_thresh) by id, then mid
//     (small_thresh <= deg < large_thresh) by id, then small (deg <
//     small_thresh) by id; small vertices are stored as a plain CSR.
//   * the stream is MSB-first; in memory it is held as 32-bit words with bit i
//     at bit 31 - i%32 of word i/32 (the reference's File::graph).
// Bit offsets are 64-bit here; the reference's reader keeps them in 32 bits.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace lpa {

struct CgrParams {
  int zeta_k = 3;         // CgrCompressor(_zeta_k = 3, ...)
  int min_itv_len = 4;    // minimum interval length
  int itv_seg_len = 256;  // interval segment length in bits (0: unsegmented)
  int res_seg_len = 256;  // residual segment length in bits (0: unsegmented)
};

// A CSR adjacency by vertex id.  Lists must be sorted ascending without
// duplicates (the reference encoder's gap codes assume it).
struct CsrView {
  uint64_t n = 0;
  const uint64_t *row = nullptr;  // n + 1
  const uint32_t *clm = nullptr;  // row[n]
};

struct CsrGraph {
  uint64_t n = 0;
  std::vector<uint64_t> row;  // n + 1
  std::vector<uint32_t> clm;
  CsrView view() const { return CsrView{n, row.data(), clm.data()}; }
  uint64_t m() const { return row.empty() ? 0 : row.back(); }
};

// The compressed mixed graph, exactly the content of the reference's files.
struct CgrGraph {
  uint64_t n = 0;                      // vertices
  uint64_t n_c = 0;                    // compressed vertices (deg >= small_thresh)
  uint64_t n_large = 0;                // compressed vertices with deg >= large_thresh
  uint64_t total_bits = 0;             // stream length in bits
  std::vector<uint32_t> words;         // stream, big-endian 32-bit words (+ zero tail)
  std::vector<uint64_t> offsets;       // n_c + 1 bit offsets; offsets[0] = 0
  std::vector<uint32_t> vertices;      // n positions -> vertex id
  std::vector<uint32_t> small_graph;   // small CSR neighbours
  std::vector<uint32_t> small_offset;  // n - n_c + 1 (empty when n == n_c)
  int small_thresh = 0;
  int large_thresh = 128;
  uint64_t m_small() const { return small_graph.size(); }
};

// Encode a CSR with the reference's parameters.  `threads` <= 0 uses all
// hardware threads.  Throws std::invalid_argument on unsupported input.
void cgr_encode(const CsrView &g, const CgrParams &p, int small_thresh, int large_thresh,
                CgrGraph &out, int threads = 0);

// The same encoding on a GPU (byte-identical output): the per-vertex bit
// sizing and writing run one thread per compressed vertex on `device`; the
// position order, offsets prefix sum and small CSR stay on the host.  Only
// the reference parameters (3, 4, 256, 256).  Throws std::invalid_argument on
// unsupported input and std::runtime_error on a CUDA failure.
void cgr_encode_gpu(const CsrView &g, const CgrParams &p, int small_thresh, int large_thresh, CgrGraph &out,
                    int device = 0);

// Bits one vertex occupies (same parameters); used by tests and planners.
uint64_t cgr_vertex_bits(const uint32_t *nbrs, uint64_t deg, uint32_t node, const CgrParams &p);

// The reference's on-disk files: <base>.graph (bytes), <base>.offset (text:
// count, then cumulative end bit offsets), <base>.vertices.bin (int32),
// <base>.graph.small.bin / <base>.offset.small.bin (int32, only when the small
// CSR is non-empty).
void cgr_write_files(const CgrGraph &g, const std::string &base);
// Reads them back (64-bit offsets).  n is vertices.size().  Throws
// std::runtime_error on a missing or malformed file.
void cgr_read_files(const std::string &base, int small_thresh, CgrGraph &out);

// Reference .row / .clm files (uint32 arrays).
void csr_write_files(const CsrGraph &g, const std::string &base);
void csr_read_files(const std::string &base, CsrGraph &out);

// Edge-list ingest with the reference's semantics (src/file.cpp:115-195):
// whitespace-separated "u v" pairs, n = max id + 1, list of u gets v and, when
// one_way, list of v gets u; lists sorted (not de-duplicated).
void read_edge_list(const std::string &path, bool one_way, CsrGraph &out, int threads = 0);

// Sort every list and drop duplicates (and self loops when drop_loops).
void csr_normalize(CsrGraph &g, bool drop_loops, int threads = 0);

}  // namespace lpa
