// Batched personalised PageRank (many teleport vectors, one SpMM per sweep).
#pragma once

#include "graph.cuh"

namespace knb {

struct BatchParams {
  double damping = 0.85;
  bool directed = true;
  bool weighted = false;
  int dangling = 0;
  int loops = 0;
  double tol = 1e-12;
  int64_t max_iter = 10000;
  int precision = 0;        // 0 FP64, 1 mixed
  uint32_t B = 0;           // number of vectors
  bool on_device = false;   // personalization and out are device pointers
  double switch_factor = 8192;
  double switch_floor = 2e-6;
};

struct BatchInfo {
  double seconds = 0;
  int64_t sweeps = 0;               // batch sweeps (SpMM launches)
  int64_t sweeps_fp32 = 0;
  int64_t column_iterations = 0;    // sum over vectors of their own iteration counts
  int64_t column_iterations_fp32 = 0;  // of which in FP32 sweeps
  int64_t max_column_iterations = 0;
  int kernel_launches = 0;
  int refined = 0;                  // 1: the FP64 phase was an anchor and refinement sweeps
  double sweep_seconds = 0;         // device time of the sweep loops alone
};

// personalization and out are column-major n x B (vector c at c * n).
void pagerank_batch(GraphHandleImpl& g, const BatchParams& p, const double* personalization,
                    double* out, BatchInfo* info, cudaStream_t s);

}  // namespace knb
