// Reference harness for label propagation: runs RabbitBin's own
// cluster_by_propagation on the host.
//
// TEST INFRASTRUCTURE ONLY.  Like ref_shim.cpp this translation unit is the
// checker, never the product; it goes into oracle/_ref/librbref.so.
//
// oracle/build.py cuts out, verbatim and at build time (never committed):
//   * src/impl/rb_cluster.cpp:3-93    the chi-squared tail, the score rules
//                                     (RABBIT_LPA_SCORE) and LPA_SCORE_EPS;
//   * src/impl/rb_cluster.cpp:336-740 the CSR view and cluster_by_propagation;
//   * src/rabbitbin.cpp:5600-5622     the incidence build (clamp, lists,
//                                     neighbour-id order);
//   * src/rabbitbin.cpp:5643-5645     the node order (std::shuffle with
//                                     std::default_random_engine(seed)).
// What this file adds: the reference Graph's members those lines touch
// (src/rabbitbin.h:264-301), the LOG macro of src/rabbitbin.h:95, stubs for
// the Louvain and multilevel variants (reached only under RABBIT_CLUSTER),
// and one C entry point.  The score rule is read from RABBIT_LPA_SCORE when
// the library loads, and RABBIT_PAR_LPA at each call, as in the reference.
#include <algorithm>
#include <array>
#include <atomic>
#include <cassert>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <limits>
#include <numeric>
#include <random>
#include <stdexcept>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include <omp.h>

using std::cerr;
using std::endl;

typedef float StoredDistance;
using GraphNodeId = uint32_t;
using GraphEdgeId = uint32_t;
#define LOG log

namespace {

struct Graph {
  size_t n = 0;
  std::vector<GraphNodeId> from, to;
  std::vector<std::vector<GraphEdgeId>> incs;
  std::vector<StoredDistance> edgeScore;
  size_t getNodeCount() { return n; }
  size_t getEdgeCount() { return from.size(); }
  void requireCompactEdgeIds() const {
    if (from.size() > (size_t)std::numeric_limits<GraphEdgeId>::max())
      throw std::length_error("graph exceeds the 32-bit edge-ID capacity");
  }
  GraphNodeId getOtherNode(size_t e, size_t v) const { return from[e] == v ? to[e] : from[e]; }
};

int cluster_by_louvain(Graph &, std::vector<size_t> &, unsigned, double) { abort(); }
void fisher_super_merge(Graph &, std::vector<size_t> &, const std::vector<StoredDistance> &,
                        double, int) {
  abort();
}

#include "frag_lpa_rules.inc"   // src/impl/rb_cluster.cpp:3-93
#include "frag_lpa.inc"         // src/impl/rb_cluster.cpp:336-740

}  // namespace

extern "C" {

// Labels of n nodes after the reference's label propagation on the edge list
// (from, to, edgeScore); order_in (optional) replaces the seeded node order.
// Returns 0, or 1 when the reference would have exited (negative score).
int ref_label_propagation(int64_t n_nodes, int64_t n_edges, const uint32_t *from,
                          const uint32_t *to, const float *score, unsigned long long seed_in,
                          const uint32_t *order_in, uint32_t *membership_out, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  for (int64_t e = 0; e < n_edges; ++e)
    if (score[e] < 0.0f) return 1;
  Graph g;
  g.n = (size_t)n_nodes;
  g.from.assign(from, from + n_edges);
  g.to.assign(to, to + n_edges);
  g.edgeScore.assign(score, score + n_edges);
  const size_t nobs = (size_t)n_nodes;
  {
#include "frag_incidence.inc"   // src/rabbitbin.cpp:5600-5622
  }
  const unsigned long long seed = seed_in;
#include "frag_node_order.inc"  // src/rabbitbin.cpp:5643-5645
  if (order_in)
    for (size_t i = 0; i < nobs; ++i) node_order[i] = order_in[i];
  std::vector<size_t> membership;
  cluster_by_propagation(g, membership, node_order);
  for (size_t i = 0; i < nobs; ++i)
    membership_out[i] = membership.size() == nobs ? (uint32_t)membership[i] : (uint32_t)i;
  return 0;
}

// The seeded node order alone (src/rabbitbin.cpp:5643-5645).
void ref_lpa_node_order(int64_t n_nodes, unsigned long long seed_in, uint32_t *out) {
  const size_t nobs = (size_t)n_nodes;
  const unsigned long long seed = seed_in;
#include "frag_node_order.inc"
  for (size_t i = 0; i < nobs; ++i) out[i] = (uint32_t)node_order[i];
}

}  // extern "C"
