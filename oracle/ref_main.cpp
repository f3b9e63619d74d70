// Test-infrastructure driver for the reference CPU compressor.
//
// This file is part of the oracle, not of the product.  It is compiled
// together with the reference's own, unmodified `src/compressor.cpp` and
// `src/file.cpp` (see oracle/Makefile) into oracle/_ref/cgr_ref, and is used
// only by the golden-fixture generator and by tests to pin the format.
//
// Usage: cgr_ref <edge_list> <one_way 0|1> <small_node_thresh>
//   Runs the reference ingest + compressor exactly as the reference drivers do
//   (File::write_binary, src/file.cpp:76-95: CgrCompressor(3,4,256,256,one_way),
//   compresswithcost(), write_cgr(path, sms, 128), then .row/.clm) and writes
//   <edge_list>.{graph,offset,vertices.bin,row,clm[,graph.small.bin,offset.small.bin]}.
//   Prints "compress_seconds <s>" (the reference's own compresswithcost()).
//
// File::write_binary is private in the reference header; the reference's only
// public entry (File::load_graph) aborts when the small CSR is empty, so the
// private member is reached by widening access for this translation unit.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#define private public
#include "file.h"
#undef private
#include "compressor.h"

int main(int argc, char **argv) {
  if (argc != 4) {
    std::fprintf(stderr, "usage: %s <edge_list> <one_way 0|1> <small_node_thresh>\n", argv[0]);
    return 2;
  }
  std::string path = argv[1];
  bool one_way = std::atoi(argv[2]) != 0;
  int sms = std::atoi(argv[3]);
  File f(path, true, one_way, sms);
  f.write_binary();
  return 0;
}
