// PageRank of caller-supplied edge weights and its adjoint (edge gradients).
#pragma once

#include "graph.cuh"
#include "pagerank.cuh"

namespace knb {

struct AdjointParams {
  double damping = 0.85;
  bool directed = true;
  int dangling = 0;
  int loops = 0;
  const double* personalization = nullptr;  // device, n values or null
  double tol = 1e-12;                       // on ||lambda_k+1 - lambda_k||_1 / max(1, ||g||_1)
  int64_t max_iter = 10000;
};

struct AdjointInfo {
  int64_t iterations = 0;
  double change = 0;
  double seconds = 0;
  int kernel_launches = 0;
};

// PageRank with weights d_w (device, input edge order); scores to d_out.
void pagerank_weights(GraphHandleImpl& g, const double* d_w, const PagerankParams& prm,
                      double* d_out, PagerankInfo* info, cudaStream_t s);

// dL/dw into d_gw (m values, input edge order) for dL/dx = d_gx at the
// PageRank d_x of weights d_w; the adjoint vector to d_lambda if not null.
void pagerank_grad(GraphHandleImpl& g, const double* d_w, const double* d_x, const double* d_gx,
                   const AdjointParams& prm, double* d_gw, double* d_lambda, AdjointInfo* info,
                   cudaStream_t s);

}  // namespace knb
