// ./method dataset if_compressed if_directed threshold output_file
//
// The reference driver's command line and output (baselines/novaplus/
// novaplus.cu:29-107): positional arguments with the same defaults when
// argc != 6, the per-iteration "%d: %f (ms), updated %d" lines, the final
// "f1: <s>(s),f2: <ms>" line and the appended output-file record.  It runs the
// B200 propagator for 20 iterations.  Invoked under a name containing "cglp"
// it forces the two-pass decode-then-propagate variant and writes "cglp file: "
// records (baselines/cglp/cglp.cu:84).
//
// Environment (optional): LPA_CMS_THRESHOLD (default 128, include/decoder.cuh:51),
// LPA_ITERS (default 20), LPA_DISPATCH (fixed | learned), LPA_EARLY_EXIT (0|1).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>

#include "lpa/file.h"
#include "lpa/graph.h"
#include "lpa/label_propagator.h"

int main(int argc, char *argv[]) {
  using namespace lpa;
  bool compress = true;
  bool edge_stored_once = true;
  int small_node_thresh = 32;
  std::string inputfile, outputfile;
  if (argc == 6) {
    inputfile = argv[1];
    compress = std::atoi(argv[2]) != 0;
    edge_stored_once = std::atoi(argv[3]) != 0;
    small_node_thresh = std::atoi(argv[4]);
    outputfile = argv[5];
  } else {
    inputfile = "../../../dataset/dblp/dblp0/com-dblp.ungraph.txt";
    compress = true;
    edge_stored_once = true;
    small_node_thresh = 0;
    outputfile = "./output.txt";
  }
  const std::string prog = argv[0];
  const bool cglp = prog.find("cglp") != std::string::npos;

  PropagatorOptions opts;
  if (const char *e = std::getenv("LPA_CMS_THRESHOLD")) opts.cms_threshold = uint32_t(std::strtoul(e, nullptr, 10));
  int niter = 20;
  if (const char *e = std::getenv("LPA_ITERS")) niter = std::atoi(e);
  if (const char *e = std::getenv("LPA_DISPATCH")) opts.dispatch = std::strcmp(e, "learned") == 0 ? LPA_DISPATCH_LEARNED : LPA_DISPATCH_FIXED;
  if (const char *e = std::getenv("LPA_EARLY_EXIT")) opts.early_exit = std::atoi(e) != 0;
  if (cglp) {
    opts.dispatch = LPA_DISPATCH_FORCE;
    opts.force_variant = LPA_VARIANT_TWO_PASS;
  }

  try {
    File f(inputfile, compress, edge_stored_once, small_node_thresh);
    f.load_graph();
    std::cout << "Input graph check:\n"
              << "clm_size(csr_all_nodes): " << f.clm.size() << "\n"
              << "row_size(csr_all_nodes): " << f.row.size() << "\n"
              << "graph_size(cgr_big+mid_nodes): " << f.graph.size() << "\n"
              << "offset_size(cgr_big+mid_nodes): " << f.offset.size() << "\n"
              << "vertices size(all_nodes): " << f.vertices.size() << "\n"
              << "small graph length: " << f.small_graph.size() << "\n"
              << "small offset length: " << f.small_offset.size() << std::endl;
    using Vertex = uint32_t;
    using Edge = uint32_t;
    std::shared_ptr<CGRGraph<Vertex, Edge>> graph;
    if (compress) {
      graph = std::make_shared<CGRGraph<Vertex, Edge>>(f.clm, f.row, f.graph, f.offset, f.small_graph,
                                                        f.small_offset, f.vertices, small_node_thresh);
    } else {
      // uncompressed run: every vertex goes through the CSR path
      std::vector<Vertex> ids(f.row.size() - 1), words;
      for (size_t i = 0; i < ids.size(); i++) ids[i] = Vertex(i);
      std::vector<uint64_t> no_offsets;
      graph = std::make_shared<CGRGraph<Vertex, Edge>>(f.clm, f.row, words, no_offsets, f.clm, f.row, ids,
                                                        small_node_thresh);
    }
    std::unique_ptr<LabelPropagator<Vertex, Edge>> propagator =
        make_unique_ptr<B200Propagator<Vertex, Edge>>(graph, opts);
    std::pair<double, double> result = propagator->run(niter);
    const double f1 = result.first, f2 = result.second;
    std::cout << "f1: " << f1 / 1000 << "(s)"
              << ",f2: " << f2 << std::endl;
    if (argc != 1) {
      std::ofstream writefile(outputfile, std::ios::app);
      writefile << (cglp ? "cglp file: " : "nova file: ") << inputfile << std::endl
                << " running time: " << f1 / 1000 << "thre: " << small_node_thresh << std::endl;
      writefile << "~~~~~" << std::endl;
    }
  } catch (const std::exception &e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
