// Graph containers with the reference's names and constructors
// (include/graph.h:17-115).  CGRGraph keeps its bit offsets as 64-bit values.
#pragma once
#include <cstdint>
#include <iostream>
#include <memory>
#include <utility>
#include <vector>

namespace lpa {

template <typename T, typename... Args>
std::unique_ptr<T> make_unique_ptr(Args &&...args) {
  return std::unique_ptr<T>(new T(std::forward<Args>(args)...));
}

template <typename V, typename E>
class Graph {
 public:
  Graph() = default;
  Graph(V _n, E _m) : n(_n), m(_m) {}
  virtual ~Graph() = default;
  V n;  // number of vertices
  E m;  // number of stored arcs
};

template <typename V, typename E>
class CSRGraph : public Graph<V, E> {
 public:
  CSRGraph() = default;
  CSRGraph(std::vector<E> _neighbors, std::vector<V> _offsets)
      : Graph<V, E>(V(_offsets.size() - 1), E(_neighbors.size())),
        neighbors(std::move(_neighbors)),
        offsets(std::move(_offsets)) {}
  std::vector<V> neighbors;
  std::vector<E> offsets;
};

// The mixed graph: compressed vertices in the bitstream, small vertices as a
// CSR, plus the full CSR (the reference keeps it for degrees and tests).
template <typename V, typename E>
class CGRGraph : public Graph<V, E> {
 public:
  CGRGraph() = default;
  CGRGraph(std::vector<V> &_csr_neighbors, std::vector<E> &_csr_offsets, std::vector<V> &_cgr_neighbors,
           std::vector<uint64_t> &_cgr_offsets, std::vector<V> &_csr_small_neighbors,
           std::vector<E> &_csr_small_offsets, std::vector<V> &_vertices, int sns)
      : Graph<V, E>(V(_vertices.size()), E(_csr_neighbors.size())),
        csr_neighbors(_csr_neighbors),
        csr_offsets(_csr_offsets),
        cgr_neighbors(_cgr_neighbors),
        cgr_offsets(_cgr_offsets),
        csr_small_neighbors(_csr_small_neighbors),
        csr_small_offsets(_csr_small_offsets),
        vertices(_vertices),
        small_node_thresh(sns) {
    n_small = _csr_small_offsets.empty() ? 0 : int(_csr_small_offsets.size() - 1);
    m_small = int(_csr_small_neighbors.size());
  }
  std::vector<V> csr_neighbors;
  std::vector<E> csr_offsets;
  std::vector<V> cgr_neighbors;      // bitstream words
  std::vector<uint64_t> cgr_offsets;  // n_c + 1 bit offsets
  std::vector<V> csr_small_neighbors;
  std::vector<E> csr_small_offsets;
  std::vector<V> vertices;
  int small_node_thresh = 0;
  int n_small = 0;
  int m_small = 0;
};

template <typename V, typename E>
class CGRGraphPure : public Graph<V, E> {
 public:
  CGRGraphPure() = default;
  CGRGraphPure(std::vector<V> &_csr_neighbors, std::vector<E> &_csr_offsets, std::vector<V> &_cgr_neighbors,
               std::vector<uint64_t> &_cgr_offsets, std::vector<V> &_vertices)
      : Graph<V, E>(V(_vertices.size()), E(_csr_neighbors.size())),
        csr_neighbors(_csr_neighbors),
        csr_offsets(_csr_offsets),
        cgr_neighbors(_cgr_neighbors),
        cgr_offsets(_cgr_offsets),
        vertices(_vertices) {}
  std::vector<V> csr_neighbors;
  std::vector<E> csr_offsets;
  std::vector<V> cgr_neighbors;
  std::vector<uint64_t> cgr_offsets;
  std::vector<V> vertices;
};

}  // namespace lpa
