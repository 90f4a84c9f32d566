// Eigenvector centrality on the device: power iteration for directed
// matrices and thick-restart Lanczos for symmetric ones.
#pragma once

#include <vector>

#include "graph.cuh"

namespace knb {

struct EigenParams {
  int mode = 2;       // 1 out, 2 in, 3 all
  bool weighted = false;
  int scale = 0;      // 0 max, 1 unit
  int loops = 0;      // 0 twice, 1 once, 2 ignore
  double tol = 1e-12;
  int64_t max_iter = 10000;
  int precision = 0;  // 0 FP64, 1 FP32 products with FP64 basis
};

struct EigenResult {
  double eigenvalue = 0;
  int64_t matvecs = 0;
  int64_t matvecs_fp32 = 0;
  bool connected = true;
  double seconds = 0;
  int kernel_launches = 0;
};

// Component labels (0..count-1) and sizes.
struct Comps {
  std::vector<uint32_t> membership;
  std::vector<uint32_t> sizes;
  size_t count() const { return sizes.size(); }
};
// Weak components of the handle's edges (device union-find; each
// component's label follows its smallest node).
Comps weak_components(GraphHandleImpl& g, cudaStream_t s);
// Strong components of the handle's edges on the device, labelled in order
// of smallest node. With w (device, one value per edge) only edges with
// w > 0 take part; with `both` every edge also counts reversed.
Comps strong_components(GraphHandleImpl& g, const double* w, bool both, int* launches,
                        cudaStream_t s);

// Writes n scores to `out` (host). Throws knb::Error on failure.
void eigenvector(GraphHandleImpl& g, const EigenParams& p, double* out, EigenResult* r,
                 cudaStream_t s);

// Hubs and authorities (reference: crates/engine/src/metrics/spectral.rs:
// 676-903): blocks of the bipartite hub-authority graph, bounds on each
// block's leading value, thick-restart Lanczos on A_b^T A_b from A_b^T 1
// for the blocks that may hold the largest, ties combined. Writes n hub and
// n authority scores (host), the largest eigenvalue of A^T A and whether
// the leading singular value is simple.
struct HitsParams {
  bool weighted = false;
  int loops = 0;   // 0 twice, 1 once, 2 ignore
  int scale = 0;   // 0 largest 1, 1 sum 1, 2 unit norm
  double tol = 1e-12;
  int64_t max_iter = 10000;
};
void hits(GraphHandleImpl& g, const HitsParams& p, double* hubs, double* auths, double* value,
          int* unique, cudaStream_t s);

// The device solver of the projected Lanczos problems (one warp, EISPACK
// tred2 + tql2 order; reference: crates/engine/src/linalg.rs:478-720) on a
// host matrix: a is row-major symmetric n x n (n <= 20); eigenvalues
// ascending, eigenvectors in the columns of vecs (row-major). Returns false
// if the QL iteration does not converge.
bool symmetric_eigen_device(const double* a, int n, double* vals, double* vecs, cudaStream_t s);

// Newman's leading eigenvector communities of an undirected graph with at
// most 3000 nodes (crates/engine/src/metrics/partition/leading_eigen.rs):
// n labels by first appearance, the modularity on the input network and the
// number of divisions.
void leading_eigen(GraphHandleImpl& g, bool weighted, int64_t* membership, double* q,
                   int64_t* splits, int* launches, cudaStream_t s);

// FP64 products y = A x on merge-path warp tiles over the rows of `v`
// (offsets from 0) with the partition build_partition makes for
// product_tile() items per tile; the scratch grows on first use.
struct ProductScratch {
  DevBuf<double> carry, head, part1, part2;
};
uint32_t product_tile();
void product64(const OpView<double>& v, const Partition& P, const double* x, double* y,
               ProductScratch& sc, cudaStream_t s);

}  // namespace knb
