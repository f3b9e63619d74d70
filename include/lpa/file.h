// File: ingest + compressed-file cache, the reference's interface
// (include/file.h:28-76, src/file.cpp:9-276) over the native format layer.
//
// Same constructor, load_graph() and public vectors.  One deliberate change:
// `offset` holds 64-bit bit offsets (the reference parses them as uint32,
// src/file.cpp:242-259, which overflows past 2^32 bits = 512 MiB of stream).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace lpa {

using Uint = uint32_t;

class File {
 public:
  // _one_way: the edge list stores each edge once; reverse arcs are added.
  // sms: small-node threshold; vertices with degree < sms stay uncompressed.
  File(const std::string _file_name, bool _compress, bool _one_way, int sms = 32);

  // Loads the graph, first writing the cache files (.graph .offset
  // .vertices.bin .row .clm [.graph.small.bin .offset.small.bin]) when any of
  // .graph/.offset/.row (or .clm for an uncompressed load) is missing.
  // Throws std::runtime_error on unreadable or malformed files.
  void load_graph();

  // csr (all vertices, by id)
  std::vector<Uint> clm;
  std::vector<Uint> row;
  // cgr (compressed vertices, in position order)
  std::vector<Uint> graph;        // big-endian 32-bit words of the bitstream
  std::vector<uint64_t> offset;   // n_c + 1 bit offsets (64-bit)
  std::vector<Uint> vertices;     // position -> vertex id
  // small vertices kept as CSR
  std::vector<Uint> small_graph;
  std::vector<Uint> small_offset;
  Uint vertex_num = 0;
  int small_node_thresh;

  // Number of compressed vertices (offset.size() - 1).
  uint64_t compressed_num() const { return offset.empty() ? 0 : offset.size() - 1; }

 private:
  std::string file_name;
  bool compress;
  bool one_way;
  bool has_small;

  void write_binary();
  void load_compress_graph();
};

}  // namespace lpa
