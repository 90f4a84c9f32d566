// Graphs from a frame's resolved edge table, on the device: the last steps of
// the reference's frame path (crates/engine/src/frame/build.rs), which turn
// validated tables into graphs.
#pragma once

#include <vector>

#include "common.cuh"

namespace knb {

// A resolved edge table: endpoint node indices of every row (host, m
// values each), optional weights, optional missing flags (rows marked 1 are
// unobserved and left out of every graph), over n nodes.
struct FrameTable {
  int64_t n = 0;
  int64_t m = 0;
  const int64_t* src = nullptr;
  const int64_t* tgt = nullptr;
  const double* weights = nullptr;
  const uint8_t* missing = nullptr;
};

// The edges of a graph to build, in their final order, on the device.
struct FrameEdges {
  uint32_t n = 0;              // nodes of the graph
  uint64_t m = 0;              // its edges
  DevBuf<uint32_t> src, tgt;   // m each
  DevBuf<double> w;            // m, when the table has weights
  DevBuf<uint32_t> rows;       // m: the table row of each edge
  DevBuf<uint32_t> node_ids;   // packed egos: the table's node index of each node
  std::vector<int64_t> node_offsets;  // packed egos: ego k on [off[k], off[k + 1])
};

// graph_of (build.rs:106-121): the observed rows in row order over all n
// nodes. Throws knb::Error naming the first bad row.
void frame_observed(const FrameTable& t, FrameEdges* out, cudaStream_t s);

// Every ego's subgraph (build.rs:153-194, 220-238) packed back to back:
// ego k keeps the nodes i with node_ego[i] == k, ascending, and the observed
// rows e with edge_ego[e] == k whose endpoints both belong to ego k, in row
// order; egos follow one another in label order (-1 or any value outside
// 0..egos-1 marks a node or row of no ego).
void frame_egos(const FrameTable& t, const int64_t* node_ego, const int64_t* edge_ego,
                int64_t egos, FrameEdges* out, cudaStream_t s);

}  // namespace knb
