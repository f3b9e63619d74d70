// CgrCompressor (include/lpa/compressor.h) over the parallel encoder.
#include "lpa/compressor.h"

#include <chrono>
#include <iostream>
#include <stdexcept>

namespace lpa {

CgrCompressor::CgrCompressor(int _zeta_k, int _min_itv_len, int _itv_seg_len, int _res_seg_len, int _one_way)
    : one_way_storage(_one_way != 0) {
  params_.zeta_k = _zeta_k;
  params_.min_itv_len = _min_itv_len;
  params_.itv_seg_len = _itv_seg_len;
  params_.res_seg_len = _res_seg_len;
}

bool CgrCompressor::load_graph(const std::string &file_path) {
  read_edge_list(file_path, one_way_storage, graph_);
  return true;
}

void CgrCompressor::set_graph(CsrGraph g) { graph_ = std::move(g); }

void CgrCompressor::compress() {
  cgr_encode(graph_.view(), params_, 0, 128, cgr_);
  std::cout << "compress done" << std::endl;
}

double CgrCompressor::compresswithcost() {
  auto t0 = std::chrono::steady_clock::now();
  cgr_encode(graph_.view(), params_, 0, 128, cgr_);
  auto t1 = std::chrono::steady_clock::now();
  std::cout << "compress done" << std::endl;
  return std::chrono::duration<double>(t1 - t0).count();
}

bool CgrCompressor::write_cgr(const std::string &file_path, int small_node_thresh, int large_node_thresh) {
  if (cgr_.small_thresh != small_node_thresh || cgr_.large_thresh != large_node_thresh || cgr_.n != graph_.n ||
      cgr_.offsets.empty())
    cgr_encode(graph_.view(), params_, small_node_thresh, large_node_thresh, cgr_);
  cgr_write_files(cgr_, file_path);
  return true;
}

int CgrCompressor::get_significant_bit(size_type x) {
  if (x <= 0) throw std::invalid_argument("get_significant_bit: x must be positive");
  return 63 - __builtin_clzll(uint64_t(x));
}

void CgrCompressor::encode(bits &bit_array, size_type x, int len) {
  for (int i = len - 1; i >= 0; i--) bit_array.push_back((x >> i) & 1L);
}

void CgrCompressor::encode_gamma(bits &bit_array, size_type x) {
  x++;
  int len = get_significant_bit(x);
  encode(bit_array, 1, len + 1);
  encode(bit_array, x, len);
}

void CgrCompressor::encode_zeta(bits &bit_array, size_type x) {
  if (params_.zeta_k == 1) {
    encode_gamma(bit_array, x);
    return;
  }
  x++;
  int len = get_significant_bit(x);
  int h = len / params_.zeta_k;
  encode(bit_array, 1, h + 1);
  encode(bit_array, x, (h + 1) * params_.zeta_k);
}

size_type CgrCompressor::gamma_size(size_type x) { return 2 * get_significant_bit(x + 1) + 1; }

size_type CgrCompressor::zeta_size(size_type x) {
  if (params_.zeta_k == 1) return gamma_size(x);
  int h = get_significant_bit(x + 1) / params_.zeta_k;
  return size_type(h + 1) * (params_.zeta_k + 1);
}

uint64_t CgrCompressor::node_bits(size_type node) const {
  if (node < 0 || uint64_t(node) >= graph_.n) throw std::out_of_range("node_bits: node out of range");
  const uint64_t b = graph_.row[node], e = graph_.row[node + 1];
  return cgr_vertex_bits(graph_.clm.data() + b, e - b, uint32_t(node), params_);
}

}  // namespace lpa
