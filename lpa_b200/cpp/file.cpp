// File (include/lpa/file.h): the reference's ingest and cache semantics
// (src/file.cpp:9-276) over the native format layer.
#include "lpa/file.h"

#include <sys/stat.h>

#include <cstdio>
#include <iostream>
#include <stdexcept>

#include "lpa/cgr_format.h"

namespace lpa {

namespace {
bool exists(const std::string &p) {
  struct stat st;
  return ::stat(p.c_str(), &st) == 0;
}
}  // namespace

File::File(const std::string _file_name, bool _compress, bool _one_way, int sms)
    : small_node_thresh(sms), file_name(_file_name), compress(_compress), one_way(_one_way) {
  has_small = sms != 0;
  std::cout << "graph file: " << _file_name << "\ncompressed: " << _compress << "\nsmall-node CSR: " << has_small
            << "\n";
  if (has_small) std::cout << "small-node threshold: " << sms << "\n";
  std::cout << "edge list stores each edge once: " << _one_way << "\n";
}

void File::write_binary() {  // src/file.cpp:76-95
  CsrGraph csr;
  read_edge_list(file_name, one_way, csr);
  if (compress) {
    CgrParams p;  // CgrCompressor(3, 4, 8 * 32, 8 * 32, one_way)
    CgrGraph cgr;
    cgr_encode(csr.view(), p, small_node_thresh, 128, cgr);
    cgr_write_files(cgr, file_name);
  }
  csr_write_files(csr, file_name);
}

void File::load_compress_graph() {
  CgrGraph g;
  cgr_read_files(file_name, small_node_thresh, g);
  graph.assign(g.words.begin(), g.words.end());
  offset = std::move(g.offsets);
  vertices = std::move(g.vertices);
  if (has_small) {
    small_graph = std::move(g.small_graph);
    small_offset = std::move(g.small_offset);
  }
}

void File::load_graph() {  // src/file.cpp:24-74
  std::cout << "load graph : " << file_name << std::endl;
  const std::string csr_graph = file_name + ".clm", csr_offset = file_name + ".row";
  if (compress) {
    if (!exists(file_name + ".graph") || !exists(file_name + ".offset") || !exists(csr_offset)) write_binary();
    load_compress_graph();
  } else if (!exists(csr_graph)) {
    write_binary();
  }
  CsrGraph csr;
  csr_read_files(file_name, csr);
  row.assign(csr.row.begin(), csr.row.end());
  clm = std::move(csr.clm);
  if (compress) {
    vertex_num = Uint(vertices.size());
  } else {
    vertex_num = Uint(row.size() - 1);
  }
}

}  // namespace lpa
