// PageRank on every graph of a packed batch (block-diagonal handle).
#pragma once

#include "graph.cuh"

namespace knb {

struct EgoInput {
  uint32_t count = 0;
  const int64_t* node_offsets = nullptr;  // count + 1, host
  double damping = 0.85;
  bool directed = true;
  bool weighted = false;
  int dangling = 0;
  int loops = 0;
  double tol = 1e-12;
  int64_t max_iter = 10000;
  const double* personalization = nullptr;  // host, n values or null
  bool out_on_device = false;
  int64_t* iterations_out = nullptr;        // host, count values or null
};

struct EgoResult {
  double seconds = 0;
  int threads = 0;
  int64_t total_iterations = 0;
  int64_t max_iterations = 0;
  int instantiations = 0;  // times the operator's launch graph has been instantiated
  int cluster = 1;         // CTAs per cluster that split the large graphs (1: none split)
  int32_t split_graphs = 0;  // graphs split over a cluster
  double change = 0;         // a batch of one graph: its last L1 change
};

void pagerank_graphs(GraphHandleImpl& g, const EgoInput& in, double* out, EgoResult* res,
                     cudaStream_t s);
void set_ego_threads(int threads);
void set_ego_cluster(int ctas);           // 0: tuned with the threads; 1, 4 or 8
void set_ego_big_nodes(int64_t nodes);    // 0: automatic

}  // namespace knb
