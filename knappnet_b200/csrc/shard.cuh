// Row shards of one graph's PageRank, for a solve split over several GPUs by
// rows of the pull operator (one process per GPU). The reference runs the
// whole loop in one process (crates/engine/src/metrics/spectral.rs:247-280);
// split by rows, one sweep is
//   1. each rank: y_r = d (A_r z + D jump_r) + (1 - d) p_r over its rows, and
//      its partial sum t_r of y_r (fixed order), into a payload of
//      payload_len doubles (rows, padding, t_r in the last slot);
//   2. the ranks all-gather the payloads (the one exchange of a sweep);
//   3. every rank, over all n nodes from the gathered payloads: T = sum of
//      t_r in rank order, x' = y / T, change = sum |x' - x|, z = x' / out
//      (0 where out is 0) and the dangling mass D = sum of x' over those
//      nodes, all in a fixed order,
// so every rank holds the same iterate, bit for bit, and takes the same
// stopping decision without a second collective.
#pragma once

#include <memory>
#include <vector>

#include "eigen.cuh"
#include "graph.cuh"

namespace knb {

struct ShardState {
  double stuck;    // dangling mass D of the current iterate
  double change;   // L1 change of the last finished sweep
  unsigned int ticket;
  unsigned int pad;
};

// Shards hold ranges of the operator's rows renumbered by column count
// (Operator::relabeled: the values a sweep gathers most sit together, and
// each row keeps its arcs in order, so its sum is the same); iterates are in
// that numbering, and scores go back to node order when read.
//
// parts + 1 boundaries 0 = b_0 <= ... <= b_parts = n of those rows: b_k is
// the first row r with r + off[r] >= k (n + nnz) / parts, so each range
// holds about an equal share of rows plus arcs.
std::vector<int64_t> shard_bounds(Operator& op, int parts, cudaStream_t s);

struct Shard {
  Operator* op = nullptr;
  const Relabeled* rl = nullptr;  // the renumbered rows (null for n = 0)
  uint32_t n = 0, r0 = 0, r1 = 0;
  uint64_t arc0 = 0;        // the first row's first arc
  uint64_t arcs = 0;        // arcs of the shard's rows
  int parts = 1, rank = 0;
  size_t payload_len = 0;   // doubles a rank sends per sweep
  double damping = 0.85;
  bool pers = false;        // personalization given (else uniform)
  bool jump_uniform = true; // dangling mass spread uniformly
  std::vector<int64_t> bounds;
  DevBuf<int64_t> dbounds;
  DevBuf<uint32_t> off;     // the shard's row offsets, from 0
  std::unique_ptr<Partition> part;
  ProductScratch scratch;
  DevBuf<double> p;         // personalization of the shard's rows
  DevBuf<double> x, z;      // current iterate and x / out, all n nodes
  DevBuf<double> out;       // out-strengths in the renumbered order
  DevBuf<double> scores;    // the iterate in node order (shard_scores)
  DevBuf<double> part_rows, part_all;  // block partials
  DevBuf<ShardState> st;
  ShardState* hst = nullptr;  // pinned
  ~Shard();
};

// Builds rank `rank`'s shard of bounds (parts + 1 values) on operator op and
// starts it at the uniform iterate. d_pers: n device values already
// normalised, or null.
std::unique_ptr<Shard> shard_new(Operator& op, double damping, const double* d_pers,
                                 bool jump_uniform, const std::vector<int64_t>& bounds,
                                 int rank, cudaStream_t s);
// Step 1 into d_payload (payload_len doubles, device).
void shard_sweep(Shard& sh, double* d_payload, cudaStream_t s);
// Back to the uniform iterate (x = 1/n), as after shard_new.
void shard_restart(Shard& sh, cudaStream_t s);
// The current iterate in node order into out (n doubles, device or host).
void shard_scores(Shard& sh, double* out, bool out_on_device, cudaStream_t s);
// Step 3 from d_gathered (parts * payload_len doubles, rank order); returns
// the change (waits for the stream).
double shard_finish(Shard& sh, const double* d_gathered, cudaStream_t s);

}  // namespace knb
