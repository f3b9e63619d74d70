// CgrCompressor: the reference's compressor interface (include/compressor.h:
// 23-138) backed by the fast parallel, bit-identical encoder (cgr_format.h).
//
// Same constructor defaults and public entry points; the per-code helpers
// (encode_gamma, encode_zeta, append_*, gamma_size, zeta_size, int_2_nat,
// get_significant_bit) produce the same bits as the reference's.
#pragma once
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

#include "lpa/cgr_format.h"

namespace lpa {

using size_type = int64_t;
using bits = std::vector<bool>;

class CgrCompressor {
 public:
  explicit CgrCompressor(int _zeta_k = 3, int _min_itv_len = 4, int _itv_seg_len = 0, int _res_seg_len = 4 * 32,
                         int _one_way = true);

  // Reads a text edge list ("u v" per line, 64-bit ids), adding reverse arcs
  // when one_way; every list sorted (src/compressor.cpp:22-68).
  bool load_graph(const std::string &file_path);
  // Uses an in-memory CSR instead (lists sorted, no duplicates).
  void set_graph(CsrGraph g);

  // Encodes every vertex (timing only; the layout is fixed by write_cgr).
  void compress();
  // Same, returning the encoding time in seconds (src/compressor.cpp:85-100).
  double compresswithcost();
  // Writes <path>.graph, .offset, .vertices.bin and the small CSR files.
  bool write_cgr(const std::string &file_path, int small_node_thresh = 32, int large_node_thresh = 128);

  // Per-code helpers, bit for bit as the reference's.
  void encode_gamma(bits &bit_array, size_type x);
  void encode_zeta(bits &bit_array, size_type x);
  void encode(bits &bit_array, size_type x, int len);
  void append_gamma(bits &bit_array, size_type x) { encode_gamma(bit_array, x); }
  void append_zeta(bits &bit_array, size_type x) { encode_zeta(bit_array, x); }
  size_type int_2_nat(size_type x) { return x >= 0L ? x << 1 : -((x << 1) + 1L); }
  size_type gamma_size(size_type x);
  size_type zeta_size(size_type x);
  int get_significant_bit(size_type x);

  // Bits of one vertex's encoding (the reference's encode_node output size).
  uint64_t node_bits(size_type node) const;

  const CsrGraph &csr() const { return graph_; }
  const CgrGraph &cgr() const { return cgr_; }

 private:
  CgrParams params_;
  bool one_way_storage;
  CsrGraph graph_;
  CgrGraph cgr_;
};

}  // namespace lpa
