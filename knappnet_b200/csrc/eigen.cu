// Eigenvector centrality on the device (reference:
// crates/engine/src/metrics/eigenvector.rs:229-1137).
//
// - Directed matrices: power iteration on A' + I, rescaled to a largest
//   entry of 1 after every product, stopped when no entry changes by more
//   than tol (eigenvector.rs:330-374). One step is the merge-path product
//   with the shift fused into its epilogue (y = A'x + x and the block
//   maximum), the split-row kernel, and a vertex kernel that divides by the
//   maximum and reduces the infinity-norm change.
// - Symmetric matrices: per weak component, thick-restart Lanczos with full
//   reorthogonalisation (classical Gram-Schmidt with the DGKS test) and the
//   reference's constants (basis <= 20, keep 8, a convergence check every 4
//   steps, a true-residual check of every candidate; eigenvector.rs:729-878).
//   The basis, the products, the projections and the norms live on the
//   device; the DGKS decision is taken on the device, and so is the <= 20 x
//   20 projected eigenproblem at each check (one warp, EISPACK order); the
//   host reads a few scalars per check to choose the next step. Sums over vectors
//   use fixed 4096-row blocks added in a fixed order (eigenvector.rs:913-971),
//   so the results do not change from run to run.
// - Components: weak components by a concurrent union-find on the device
//   whose roots are the smallest node of each component, relabelled in order
//   of their smallest node (topography.rs:183-246); strong components (for
//   directed matrices) also on the device, by rounds of trimming, max-colour
//   propagation and backward propagation from each colour's root, labelled
//   in the order of Tarjan's first appearance (topography.rs:248-305).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <unordered_map>
#include <deque>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "eigen.cuh"

namespace knb {

// ======================================================================= components
constexpr int ET = 256;

__device__ __forceinline__ uint32_t uf_find(uint32_t* parent, uint32_t v) {
  uint32_t p = parent[v];
  while (p != v) {
    uint32_t gp = parent[p];
    if (gp != p) parent[v] = gp;  // path halving; races only shorten paths
    v = p;
    p = gp;
  }
  return v;
}

__global__ void uf_init(uint32_t* parent, uint32_t n) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    parent[v] = v;
}

// Union by smaller root with compare-and-swap: a root only ever hooks under
// a smaller root, so every final root is its component's smallest node.
__global__ void uf_union(uint32_t* parent, const uint32_t* __restrict__ src,
                         const uint32_t* __restrict__ tgt, uint64_t m) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a = uf_find(parent, src[e]), b = uf_find(parent, tgt[e]);
    while (a != b) {
      uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
      uint32_t old = atomicCAS(&parent[hi], hi, lo);
      if (old == hi) break;
      a = uf_find(parent, old);
      b = uf_find(parent, lo);
    }
  }
}

__global__ void uf_roots(uint32_t* parent, uint32_t n, uint32_t* root, uint32_t* is_root) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    uint32_t r = uf_find(parent, v);
    root[v] = r;
    is_root[v] = r == v;
  }
}

__global__ void uf_label(const uint32_t* __restrict__ root, const uint32_t* __restrict__ rank,
                         uint32_t n, uint32_t* __restrict__ label, uint32_t* __restrict__ sizes) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    uint32_t c = rank[root[v]];
    label[v] = c;
    atomicAdd(&sizes[c], 1u);
  }
}

Comps weak_components(GraphHandleImpl& g, cudaStream_t s) {
  const uint32_t n = g.n;
  DevBuf<uint32_t> parent(n), root(n), flag(n + 1), label(n);
  uf_init<<<grid_for(n, ET), ET, 0, s>>>(parent.get(), n);
  if (g.m) uf_union<<<grid_for(g.m, ET), ET, 0, s>>>(parent.get(), g.src.get(), g.tgt.get(), g.m);
  uf_roots<<<grid_for(n, ET), ET, 0, s>>>(parent.get(), n, root.get(), flag.get());
  KNB_LAUNCH("weak components");
  uint32_t k = exclusive_scan<uint32_t>(flag.get(), flag.get(), n, s);
  DevBuf<uint32_t> sizes(std::max<uint32_t>(k, 1));
  KNB_CUDA(cudaMemsetAsync(sizes.get(), 0, (size_t)std::max<uint32_t>(k, 1) * 4, s));
  uf_label<<<grid_for(n, ET), ET, 0, s>>>(root.get(), flag.get(), n, label.get(), sizes.get());
  KNB_LAUNCH("uf_label");
  Comps c;
  c.membership.resize(n);
  c.sizes.resize(k);
  KNB_CUDA(cudaMemcpyAsync(c.membership.data(), label.get(), (size_t)n * 4, cudaMemcpyDeviceToHost, s));
  if (k) KNB_CUDA(cudaMemcpyAsync(c.sizes.data(), sizes.get(), (size_t)k * 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  return c;
}

// ======================================================================= strong components (device)
// Strong components of the arcs (src[e], tgt[e]) on the device, as rounds
// over the nodes not yet assigned to a component:
//  1. trim: a node with no unassigned in-neighbour, or none out, other than
//     itself, is a component of its own (repeated to a fixed point);
//  2. colour: each node takes the largest id that reaches it through
//     unassigned nodes (max propagation along the arcs to a fixed point);
//  3. a node whose colour is its own id is the largest node of its
//     component, which is the set of nodes of that colour that reach it: a
//     path from such a node to the root never leaves the colour, so
//     propagation backwards along the arcs inside the colour finds it.
// Each round assigns at least the component of the largest unassigned id.
// Every pass is one thread per arc (the arc list is balanced whatever the
// degrees), and a pass that changes nothing ends its fixed point; passes
// are enqueued four at a time between reads of their change flags.
// Components are labelled in order of their smallest node, as Tarjan's
// labels (crates/engine/src/metrics/topography.rs:183-221).
constexpr uint32_t SCC_NONE = 0xFFFFFFFFu;

// Arcs (src[e], tgt[e]) for e < m; with w given only arcs with w[e] > 0
// take part; with `both` each arc also counts reversed. Loops never matter.
struct SccArcs {
  const uint32_t* src;
  const uint32_t* tgt;
  const double* w;
  uint64_t m;
  int both;
};

__device__ __forceinline__ bool scc_arc(const SccArcs& a, uint64_t e, const uint32_t* rep,
                                        uint32_t* u, uint32_t* v) {
  *u = a.src[e];
  *v = a.tgt[e];
  if (*u == *v) return false;
  if (a.w && !(a.w[e] > 0.0)) return false;
  return rep[*u] == SCC_NONE && rep[*v] == SCC_NONE;
}

__device__ __forceinline__ void scc_flag(bool c, unsigned int* flag) {
  if (__syncthreads_or(c) && threadIdx.x == 0) *flag = 1u;
}

__global__ void scc_trim_mark(SccArcs a, const uint32_t* __restrict__ rep, uint8_t* hasin,
                              uint8_t* hasout) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < a.m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u, v;
    if (!scc_arc(a, e, rep, &u, &v)) continue;
    if (!hasout[u]) hasout[u] = 1;
    if (!hasin[v]) hasin[v] = 1;
    if (a.both) {
      if (!hasout[v]) hasout[v] = 1;
      if (!hasin[u]) hasin[u] = 1;
    }
  }
}

// changed: some node was assigned; left: some node is still unassigned.
__global__ void scc_trim_assign(uint32_t n, uint32_t* rep, uint8_t* hasin, uint8_t* hasout,
                                unsigned int* changed, unsigned int* left) {
  bool c = false, l = false;
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    if (rep[v] != SCC_NONE) continue;
    if (!hasin[v] || !hasout[v]) {
      rep[v] = v;
      c = true;
    } else {
      l = true;
    }
    hasin[v] = 0;
    hasout[v] = 0;
  }
  scc_flag(c, changed);
  scc_flag(l, left);
}

__global__ void scc_color_init(uint32_t n, const uint32_t* __restrict__ rep, uint32_t* color) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    if (rep[v] == SCC_NONE) color[v] = v;
}

// Colours only grow, so a pass in which no thread raised one read settled
// values throughout: that pass ends the fixed point.
__global__ void scc_color_push(SccArcs a, const uint32_t* __restrict__ rep, uint32_t* color,
                               unsigned int* changed) {
  bool c = false;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < a.m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u, v;
    if (!scc_arc(a, e, rep, &u, &v)) continue;
    const uint32_t cu = color[u], cv = color[v];
    if (cv < cu) {
      atomicMax(&color[v], cu);
      c = true;
    }
    if (a.both && cu < cv) {
      atomicMax(&color[u], cv);
      c = true;
    }
  }
  scc_flag(c, changed);
}

__global__ void scc_roots(uint32_t n, const uint32_t* __restrict__ rep,
                          const uint32_t* __restrict__ color, uint8_t* mark) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    if (rep[v] == SCC_NONE) mark[v] = color[v] == v ? 1 : 0;
}

__global__ void scc_back(SccArcs a, const uint32_t* __restrict__ rep,
                         const uint32_t* __restrict__ color, uint8_t* mark, unsigned int* changed) {
  bool c = false;
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < a.m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t u, v;
    if (!scc_arc(a, e, rep, &u, &v)) continue;
    if (color[u] != color[v]) continue;
    const uint8_t mu = mark[u], mv = mark[v];
    if (!mu && mv) {
      mark[u] = 1;
      c = true;
    }
    if (a.both && mu && !mv) {
      mark[v] = 1;
      c = true;
    }
  }
  scc_flag(c, changed);
}

__global__ void scc_assign(uint32_t n, uint32_t* rep, const uint32_t* __restrict__ color,
                           const uint8_t* __restrict__ mark) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    if (rep[v] == SCC_NONE && mark[v]) rep[v] = color[v];
}

__global__ void scc_smallest(uint32_t n, const uint32_t* __restrict__ rep, uint32_t* smallest) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
    atomicMin(&smallest[rep[v]], v);
}

__global__ void scc_root_of(uint32_t n, const uint32_t* __restrict__ rep,
                            const uint32_t* __restrict__ smallest, uint32_t* root,
                            uint32_t* is_root) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    const uint32_t r = smallest[rep[v]];
    root[v] = r;
    is_root[v] = r == v;
  }
}

static Comps strong_components_device(const SccArcs& a, uint32_t n, int* launches,
                                      cudaStream_t s) {
  Comps c;
  if (n == 0) return c;
  constexpr int BATCH = 4;
  DevBuf<uint32_t> rep(n), color(n), smallest(n), root(n), flag((size_t)n + 1), label(n);
  DevBuf<uint8_t> hasin(n), hasout(n), mark(n);
  DevBuf<unsigned int> flags(2 * BATCH);
  unsigned int hf[2 * BATCH];
  KNB_CUDA(cudaMemsetAsync(rep.get(), 0xFF, (size_t)n * 4, s));
  KNB_CUDA(cudaMemsetAsync(hasin.get(), 0, n, s));
  KNB_CUDA(cudaMemsetAsync(hasout.get(), 0, n, s));
  const unsigned gn = grid_for(n, ET, 148 * 16);
  const unsigned ga = a.m ? grid_for(a.m, ET, 148 * 16) : 1;
  int nl = 0;
  // Runs `pass` (one pass, writing its change flag to flags[b]) to a fixed
  // point; returns the batch slot of the pass that changed nothing.
  auto settle = [&](auto pass) -> int {
    for (uint64_t done = 0;; done += BATCH) {
      if (done > (uint64_t)n + 2 * BATCH)
        throw Error("strong components did not settle (internal error)");
      KNB_CUDA(cudaMemsetAsync(flags.get(), 0, 2 * BATCH * 4, s));
      for (int b = 0; b < BATCH; ++b) pass(b);
      KNB_LAUNCH("strong components");
      KNB_CUDA(cudaMemcpyAsync(hf, flags.get(), 2 * BATCH * 4, cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaStreamSynchronize(s));
      for (int b = 0; b < BATCH; ++b)
        if (!hf[b]) return b;
    }
  };
  for (;;) {
    const int b = settle([&](int slot) {
      if (a.m) scc_trim_mark<<<ga, ET, 0, s>>>(a, rep.get(), hasin.get(), hasout.get());
      scc_trim_assign<<<gn, ET, 0, s>>>(n, rep.get(), hasin.get(), hasout.get(),
                                        flags.get() + slot, flags.get() + BATCH + slot);
      nl += 2;
    });
    if (!hf[BATCH + b]) break;
    scc_color_init<<<gn, ET, 0, s>>>(n, rep.get(), color.get());
    ++nl;
    settle([&](int slot) {
      scc_color_push<<<ga, ET, 0, s>>>(a, rep.get(), color.get(), flags.get() + slot);
      ++nl;
    });
    scc_roots<<<gn, ET, 0, s>>>(n, rep.get(), color.get(), mark.get());
    ++nl;
    settle([&](int slot) {
      scc_back<<<ga, ET, 0, s>>>(a, rep.get(), color.get(), mark.get(), flags.get() + slot);
      ++nl;
    });
    scc_assign<<<gn, ET, 0, s>>>(n, rep.get(), color.get(), mark.get());
    ++nl;
  }
  // label in order of each component's smallest node
  KNB_CUDA(cudaMemsetAsync(smallest.get(), 0xFF, (size_t)n * 4, s));
  scc_smallest<<<gn, ET, 0, s>>>(n, rep.get(), smallest.get());
  scc_root_of<<<gn, ET, 0, s>>>(n, rep.get(), smallest.get(), root.get(), flag.get());
  KNB_LAUNCH("strong component labels");
  const uint32_t k = exclusive_scan<uint32_t>(flag.get(), flag.get(), n, s);
  DevBuf<uint32_t> sizes(std::max<uint32_t>(k, 1));
  KNB_CUDA(cudaMemsetAsync(sizes.get(), 0, (size_t)std::max<uint32_t>(k, 1) * 4, s));
  uf_label<<<gn, ET, 0, s>>>(root.get(), flag.get(), n, label.get(), sizes.get());
  KNB_LAUNCH("uf_label");
  nl += 3;
  c.membership.resize(n);
  c.sizes.resize(k);
  KNB_CUDA(cudaMemcpyAsync(c.membership.data(), label.get(), (size_t)n * 4, cudaMemcpyDeviceToHost, s));
  if (k) KNB_CUDA(cudaMemcpyAsync(c.sizes.data(), sizes.get(), (size_t)k * 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  if (launches) *launches += nl;
  return c;
}

Comps strong_components(GraphHandleImpl& g, const double* w, bool both, int* launches,
                        cudaStream_t s) {
  SccArcs a{g.src.get(), g.tgt.get(), w, g.m, both ? 1 : 0};
  return strong_components_device(a, g.n, launches, s);
}

// ======================================================================= small kernels
// Any arc (v, j) inside one component with a positive value (a cycle of
// positive weight; eigenvector.rs:283-287).
__global__ void cyclic_arcs(OpView<double> op, const uint32_t* __restrict__ comp,
                            unsigned int* __restrict__ flag) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < op.n; v += gridDim.x * blockDim.x) {
    for (uint32_t k = op.off[v]; k < op.off[v + 1]; ++k) {
      double w = op.vals ? op.vals[k] : 1.0;
      if (w > 0.0 && comp[op.cols[k]] == comp[v]) {
        *flag = 1u;
        return;
      }
    }
  }
}

// Nodes whose column has no positive entry score 1 (eigenvector.rs:288-298).
__global__ void sink_scores(OpView<double> op, double* __restrict__ x) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < op.n; v += gridDim.x * blockDim.x)
    for (uint32_t k = op.off[v]; k < op.off[v + 1]; ++k) {
      double w = op.vals ? op.vals[k] : 1.0;
      if (w > 0.0) x[op.cols[k]] = 0.0;
    }
}

__global__ void fill_value(double* x, uint32_t n, double v) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = v;
}

// Row sum and the sum of squares with parallel entries merged
// (eigenvector.rs:566-584).
// Row sums and the sums of squares of rows with parallel entries merged
// (rows are sorted by column, so parallel entries are adjacent), one warp
// per row: lanes take 32 consecutive entries at a time; a ballot marks where
// runs of equal columns start, a segmented scan gives each run's sum at its
// last lane, and the run open at the chunk's end carries into the next.
__global__ void op_row_sums(OpView<double> op, double* __restrict__ s_out,
                            double* __restrict__ q_out) {
  const unsigned F = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < op.n; v += nw) {
    const uint32_t b = op.off[v], e = op.off[v + 1];
    double s = 0.0, q = 0.0, cacc = 0.0;
    uint32_t ccol = 0xFFFFFFFFu;  // column of the run open at the previous chunk's end
    for (uint32_t base = b; base < e; base += 32) {
      const uint32_t k = base + lane;
      const bool valid = k < e;
      const uint32_t j = valid ? op.cols[k] : 0xFFFFFFFEu;
      const double w = valid ? (op.vals ? op.vals[k] : 1.0) : 0.0;
      s += w;
      uint32_t pj = __shfl_up_sync(F, j, 1);
      if (lane == 0) pj = ccol;
      const bool start = j != pj;
      const uint32_t starts = __ballot_sync(F, start);
      // the run carried from the previous chunk ends where this chunk starts anew
      if (lane == 0 && (starts & 1u) && ccol != 0xFFFFFFFFu) q += cacc * cacc;
      const uint32_t upto = starts & (0xffffffffu >> (31 - lane));
      const int seg0 = upto ? 31 - __clz(upto) : -1;  // -1: the run continues from ccol
      double r = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double rr = __shfl_up_sync(F, r, o);
        if (lane - o >= (seg0 < 0 ? 0 : seg0)) r += rr;
      }
      if (seg0 < 0) r += cacc;
      const bool next_start = __shfl_down_sync(F, start, 1);
      if (valid && lane < 31 && k + 1 < e && next_start) q += r * r;
      const int last = (int)min(31u, e - 1 - base);
      cacc = __shfl_sync(F, r, last);
      ccol = __shfl_sync(F, j, last);
    }
    q = warp_sum(q);
    s = warp_sum(s);
    if (lane == 0) {
      if (e > b) q += cacc * cacc;
      s_out[v] = s;
      q_out[v] = q;
    }
  }
}

// Submatrix rows of `nodes` with columns renumbered by `local`
// (eigenvector.rs:589-624): lengths, then copies.
__global__ void sub_lengths(const uint32_t* __restrict__ off, const uint32_t* __restrict__ nodes,
                            uint32_t k, uint32_t* __restrict__ len) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x) {
    uint32_t v = nodes[i];
    len[i] = off[v + 1] - off[v];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) len[k] = 0;
}

// One warp per row (long rows copy at full width).
__global__ void sub_copy(OpView<double> op, const uint32_t* __restrict__ nodes, uint32_t k,
                         const uint32_t* __restrict__ local, const uint32_t* __restrict__ soff,
                         uint32_t* __restrict__ scols, double* __restrict__ s64,
                         float* __restrict__ s32) {
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < k; i += nw) {
    const uint32_t v = nodes[i];
    const uint32_t b = op.off[v], e = op.off[v + 1], o = soff[i];
    for (uint32_t q = b + lane; q < e; q += 32) {
      scols[o + q - b] = local[op.cols[q]];
      if (op.vals) {
        s64[o + q - b] = op.vals[q];
        s32[o + q - b] = (float)op.vals[q];
      }
    }
  }
}

// Submatrices that keep only the entries whose column is mapped (local[c]
// != 2^32 - 1), as SparseOp::submatrix (eigenvector.rs:589-624).
// Submatrices that keep only the entries whose column is mapped (local[c]
// != 2^32 - 1), in row order, as SparseOp::submatrix (eigenvector.rs:
// 589-624); one warp per row, kept entries compacted by ballot.
__global__ void sub_lengths_mapped(OpView<double> op, const uint32_t* __restrict__ nodes,
                                   uint32_t k, const uint32_t* __restrict__ local,
                                   uint32_t* __restrict__ len) {
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < k; i += nw) {
    const uint32_t v = nodes[i];
    uint32_t c = 0;
    for (uint32_t q = op.off[v] + lane; q < op.off[v + 1]; q += 32)
      c += local[op.cols[q]] != 0xFFFFFFFFu;
    c = warp_sum(c);
    if (lane == 0) len[i] = c;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) len[k] = 0;
}

__global__ void sub_copy_mapped(OpView<double> op, const uint32_t* __restrict__ nodes,
                                uint32_t k, const uint32_t* __restrict__ local,
                                const uint32_t* __restrict__ soff, uint32_t* __restrict__ scols,
                                double* __restrict__ s64) {
  const int lane = threadIdx.x & 31;
  const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < k; i += nw) {
    const uint32_t v = nodes[i];
    const uint32_t b = op.off[v], e = op.off[v + 1];
    uint32_t o = soff[i];
    for (uint32_t base = b; base < e; base += 32) {
      const uint32_t q = base + lane;
      const uint32_t c = q < e ? local[op.cols[q]] : 0xFFFFFFFFu;
      const bool keep = c != 0xFFFFFFFFu;
      const uint32_t mask = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const uint32_t pos = o + __popc(mask & ((1u << lane) - 1u));
        scols[pos] = c;
        if (s64) s64[pos] = op.vals ? op.vals[q] : 1.0;
      }
      o += __popc(mask);
    }
  }
}

__global__ void unscatter_local(const uint32_t* __restrict__ nodes, uint32_t k,
                                uint32_t* __restrict__ local) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x)
    local[nodes[i]] = 0xFFFFFFFFu;
}

__global__ void scatter_local(const uint32_t* __restrict__ nodes, uint32_t k,
                              uint32_t* __restrict__ local) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x)
    local[nodes[i]] = i;
}

__global__ void scatter_scaled(const uint32_t* __restrict__ nodes, uint32_t k,
                               const double* __restrict__ u, double factor, double* __restrict__ x) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x)
    x[nodes[i]] = u[i] * factor;
}

// ======================================================================= vector kernels
// Fixed 4096-row blocks (eigenvector.rs:913-971): one CTA per block writes
// its partial sums; the last CTA adds the partials in block order (lane l
// takes blocks l, l + 32, ...; then a fixed butterfly), so sums are
// reproducible.
constexpr int VB = 4096;
constexpr int VB_T = 256;
constexpr int MAXB = 20;  // largest basis (eigenvector.rs:730)

struct LzState {
  double coef[MAXB];   // Gram-Schmidt coefficients of the current step
  double tmp[MAXB];    // coefficients of the current pass
  double before, mid, after, beta;
  double xx, xy, value, rinf, xinf, sum;
  int32_t need2;       // second full DGKS pass needed
  int32_t breakdown;   // set at the step where beta <= 1e-12 * before
  int32_t bd_step;     // that step's j
  int32_t pad;
  uint32_t ticket;
  // the projected eigenproblem of the last check (lz_eigen)
  double theta_top;    // its largest eigenvalue
  double estimate;     // beta |s_last| of that Ritz pair (0 after a breakdown)
  int32_t eig_ok;      // 0 if the QL iteration did not converge
  int32_t eig_size;    // the projected matrix's order
};

__device__ __forceinline__ double fixed_block_sum(const double* part, uint32_t nb, int stride,
                                                  int slot) {
  // called by one full warp
  const volatile double* p = part;
  int lane = threadIdx.x & 31;
  double a = 0;
  for (uint32_t b = lane; b < nb; b += 32) a += p[(size_t)b * stride + slot];
  return warp_sum(a);
}

__device__ __forceinline__ bool lz_last(unsigned int* ticket) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x * gridDim.y - 1;
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Block-level sums of K values per thread; writes part[blockIdx * stride + s].
template <int K>
__device__ __forceinline__ void block_partials(double (&a)[K], double* part, int stride, int count) {
  __shared__ double sh[VB_T / 32][MAXB + 2];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int s = 0; s < count; ++s) {
    double v = warp_sum(a[s]);
    if (lane == 0) sh[w][s] = v;
  }
  __syncthreads();
  if (w == 0) {
    for (int s = 0; s < count; ++s) {
      double v = lane < VB_T / 32 ? sh[lane][s] : 0.0;
      v = warp_sum(v);
      if (lane == 0) part[(size_t)blockIdx.x * stride + s] = v;
    }
  }
}

// Rows of a 4096-row block held by one thread (rows t, t + 256, ...).
constexpr int VR = VB / VB_T;
// Projections per CTA of lz_project: blockIdx.y takes basis vectors
// [4y, 4y + 4), so a full pass over 20 vectors runs 5 CTAs per row block.
constexpr int LZ_PG = 4;

__host__ __device__ constexpr int lz_project_slots(int k, int mode) { return k + (mode == 0 ? 1 : 0); }
inline unsigned project_groups(int k, int mode) {
  return (unsigned)((lz_project_slots(k, mode) + LZ_PG - 1) / LZ_PG);
}

// mode 0: local pass (also computes ||w||^2 -> before); 1: full pass; 2: full
// pass 2 (skipped unless need2). Projects w on V[lo..hi). Each thread keeps its
// 16 values of w in registers and loads its 16 values of one basis vector at
// once; every dot product is summed per thread in row order, then per warp and
// CTA and over the row blocks in fixed order, as in a one-dimensional sweep.
__global__ void __launch_bounds__(VB_T)
lz_project(const double* __restrict__ V, size_t dim, int lo, int hi, const double* __restrict__ w,
           int mode, double* __restrict__ part, LzState* st, const IterState* ist) {
  if (ist && iteration_done(ist)) return;
  if (mode == 2 && !st->need2) return;
  const int K = hi - lo, slots = lz_project_slots(K, mode);
  const int s0 = blockIdx.y * LZ_PG, s1 = min(slots, s0 + LZ_PG);
  __shared__ double sh[VB_T / 32][LZ_PG];
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5;
  const size_t b0 = (size_t)blockIdx.x * VB, r1 = min(dim, b0 + VB);
  const size_t i0 = b0 + threadIdx.x;
  double wr[VR];
#pragma unroll
  for (int r = 0; r < VR; ++r) {
    const size_t i = i0 + (size_t)r * VB_T;
    wr[r] = i < r1 ? w[i] : 0.0;
  }
#pragma unroll 1
  for (int s = s0; s < s1; ++s) {
    double a = 0.0;
    if (s < K) {
      const double* vs = V + (size_t)(lo + s) * dim;
      double v[VR];
#pragma unroll
      for (int r = 0; r < VR; ++r) {
        const size_t i = i0 + (size_t)r * VB_T;
        v[r] = i < r1 ? vs[i] : 0.0;
      }
#pragma unroll
      for (int r = 0; r < VR; ++r)
        if (i0 + (size_t)r * VB_T < r1) a = fma(v[r], wr[r], a);
    } else {
#pragma unroll
      for (int r = 0; r < VR; ++r)
        if (i0 + (size_t)r * VB_T < r1) a = fma(wr[r], wr[r], a);
    }
    a = warp_sum(a);
    if (lane == 0) sh[wp][s - s0] = a;
  }
  __syncthreads();
  if (wp == 0) {
    for (int s = s0; s < s1; ++s) {
      double v = lane < VB_T / 32 ? sh[lane][s - s0] : 0.0;
      v = warp_sum(v);
      if (lane == 0) part[(size_t)blockIdx.x * (MAXB + 1) + s] = v;
    }
  }
  if (!lz_last(&st->ticket)) return;
  if (threadIdx.x < 32) {
    for (int s = 0; s < slots; ++s) {
      double v = fixed_block_sum(part, gridDim.x, MAXB + 1, s);
      if (threadIdx.x == 0) {
        if (s < K) st->tmp[s] = v;
        else st->before = sqrt(v);
      }
    }
  }
  if (threadIdx.x == 0) st->ticket = 0;
}

// w -= V[lo..hi) tmp, ||w|| into mid (mode 0) or after; coefficients added
// into coef; the DGKS decision after full passes (eigenvector.rs:997-1021).
// Each thread keeps its 16 values of w in registers and subtracts one basis
// vector at a time from all of them, in basis order.
__global__ void __launch_bounds__(VB_T)
lz_subtract(const double* __restrict__ V, size_t dim, int lo, int hi, double* __restrict__ w,
            int mode, double* __restrict__ part, LzState* st, const IterState* ist) {
  if (ist && iteration_done(ist)) return;
  if (mode == 2 && !st->need2) return;
  const int K = hi - lo;
  __shared__ double c[MAXB];
  if (threadIdx.x < K) c[threadIdx.x] = st->tmp[threadIdx.x];
  __syncthreads();
  const size_t b0 = (size_t)blockIdx.x * VB, r1 = min(dim, b0 + VB);
  const size_t i0 = b0 + threadIdx.x;
  double x[VR];
#pragma unroll
  for (int r = 0; r < VR; ++r) {
    const size_t i = i0 + (size_t)r * VB_T;
    x[r] = i < r1 ? w[i] : 0.0;
  }
  if (b0 + VB <= dim) {
#pragma unroll 1
    for (int s = 0; s < K; ++s) {
      const double* vs = V + (size_t)(lo + s) * dim + i0;
      const double cs = c[s];
      double v[VR];
#pragma unroll
      for (int r = 0; r < VR; ++r) v[r] = vs[(size_t)r * VB_T];
#pragma unroll
      for (int r = 0; r < VR; ++r) x[r] = fma(-cs, v[r], x[r]);
    }
  } else {
#pragma unroll 1
    for (int s = 0; s < K; ++s) {
      const double* vs = V + (size_t)(lo + s) * dim;
      const double cs = c[s];
#pragma unroll
      for (int r = 0; r < VR; ++r) {
        const size_t i = i0 + (size_t)r * VB_T;
        if (i < r1) x[r] = fma(-cs, vs[i], x[r]);
      }
    }
  }
  double a[1] = {0.0};
#pragma unroll
  for (int r = 0; r < VR; ++r) {
    const size_t i = i0 + (size_t)r * VB_T;
    if (i < r1) {
      w[i] = x[r];
      a[0] = fma(x[r], x[r], a[0]);
    }
  }
  block_partials<1>(a, part, 1, 1);
  if (!lz_last(&st->ticket)) return;
  if (threadIdx.x < 32) {
    double v = sqrt(fixed_block_sum(part, gridDim.x, 1, 0));
    if (threadIdx.x == 0) {
      for (int s = 0; s < K; ++s) st->coef[lo + s] += st->tmp[s];
      if (mode == 0) {
        st->mid = v;
      } else if (mode == 1) {
        st->after = v;
        bool done = v >= M_SQRT1_2 * st->mid || v == 0.0 || st->mid == st->before;
        st->need2 = done ? 0 : 1;
        if (!done) st->mid = st->before;
      } else {
        st->after = v;
      }
      st->ticket = 0;
    }
  }
}

// Start of a step: zero the coefficients.
__global__ void lz_begin(LzState* st, const IterState* ist) {
  if (ist && iteration_done(ist)) return;
  if (threadIdx.x < MAXB) st->coef[threadIdx.x] = 0.0;
  if (threadIdx.x == 0) st->need2 = 0;
}

// End of a step: coefficients into the projected matrix, beta, breakdown
// (eigenvector.rs:786-796).
__global__ void lz_end(LzState* st, IterState* ist, double* hm, int m, int j) {
  if (iteration_done(ist)) return;
  if (threadIdx.x < j + 1) {
    hm[threadIdx.x * m + j] = st->coef[threadIdx.x];
    hm[j * m + threadIdx.x] = st->coef[threadIdx.x];
  }
  if (threadIdx.x == 0) {
    double beta = st->after;
    st->beta = beta;
    bool bd = beta <= 1e-12 * st->before || isnan(beta);
    if (bd) {
      st->breakdown = 1;
      st->bd_step = j;
      ist->stopped = 1;  // later enqueued steps do nothing
    }
  }
}

// v = w / beta into basis column `col` (and its FP32 copy); hm(col, col-1).
__global__ void lz_next(double* __restrict__ V, size_t dim, int col, const double* __restrict__ w,
                        float* __restrict__ v32, double* hm, int m, const LzState* st,
                        const IterState* ist, int set_hm) {
  if (ist && iteration_done(ist)) return;
  const double beta = st->beta;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < dim;
       i += (size_t)gridDim.x * blockDim.x) {
    double v = w[i] / beta;
    V[(size_t)col * dim + i] = v;
    if (v32) v32[i] = (float)v;
  }
  if (set_hm && blockIdx.x == 0 && threadIdx.x == 0) {
    hm[col * m + col - 1] = beta;
    hm[(col - 1) * m + col] = beta;
  }
}

// x = V[0..cols) s (eigenvector.rs:1080-1092).
__global__ void lz_combine(const double* __restrict__ V, size_t dim, int cols,
                           const double* __restrict__ s, double* __restrict__ x) {
  __shared__ double c[MAXB];
  if (threadIdx.x < cols) c[threadIdx.x] = s[threadIdx.x];
  __syncthreads();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < dim;
       i += (size_t)gridDim.x * blockDim.x) {
    double o = 0.0;
    for (int l = 0; l < cols; ++l) o += c[l] * V[(size_t)l * dim + i];
    x[i] = o;
  }
}

// V[:, 0..p) = V[:, 0..cols) S (S row-major cols x p) via `out` (p vectors).
__global__ void lz_rotate(const double* __restrict__ V, size_t dim, int cols,
                          const double* __restrict__ S, int p, double* __restrict__ out) {
  __shared__ double c[MAXB * MAXB];
  for (int k = threadIdx.x; k < cols * p; k += blockDim.x) c[k] = S[k];
  __syncthreads();
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < dim;
       i += (size_t)gridDim.x * blockDim.x) {
    double o[MAXB];
    for (int q = 0; q < p; ++q) o[q] = 0.0;
    for (int l = 0; l < cols; ++l) {
      double x = V[(size_t)l * dim + i];
      for (int q = 0; q < p; ++q) o[q] += c[l * p + q] * x;
    }
    for (int q = 0; q < p; ++q) out[(size_t)q * dim + i] = o[q];
  }
}

// ------------------------------------------------------------- projected eigenproblem
// Symmetric eigensolver for the <= MAXB x MAXB projected matrix on the
// device, run by one warp: Householder tridiagonalisation with accumulated
// transformations and the implicit QL method (EISPACK tred2 / tql2; Martin,
// Reinsch and Wilkinson), as crates/engine/src/linalg.rs:478-720 restates
// them. Each matrix entry sees the same operations in the same order as in
// the sequential algorithm: lane 0 runs the scalar recurrences and every sum,
// and the warp shares only loops whose iterations touch disjoint rows or
// columns (lane r takes row r or column r). The caller loads the matrix into
// V; on return V holds the eigenvectors in its columns and d the eigenvalues
// in ascending order. Returns false if the QL iteration does not converge.
struct EigWork {
  double V[MAXB][MAXB + 1];
  double d[MAXB], e[MAXB], cs[MAXB], sn[MAXB];
  double scale, h;
  int m, done, ok, swaps[MAXB];
};

// tql2 on the tridiagonal (d, e) that tred2 leaves, rotating V's columns;
// then the eigenpairs in ascending order (selection by swaps, as EISPACK).
__device__ bool warp_tql2(EigWork& W, int n) {
  const int lane = threadIdx.x & 31;
  double (*V)[MAXB + 1] = W.V;
  double* d = W.d;
  double* e = W.e;
  double f = 0.0, tst1 = 0.0;  // lane 0's
  const double eps = DBL_EPSILON;
  if (lane == 0) {
    for (int i = 1; i < n; ++i) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    W.ok = 1;
  }
  __syncwarp();
  for (int l = 0; l < n; ++l) {
    if (lane == 0) {
      tst1 = fmax(tst1, fabs(d[l]) + fabs(e[l]));
      int m = l;
      while (m < n && !(fabs(e[m]) <= eps * tst1)) ++m;
      W.m = m;
      W.done = m > l ? 0 : 1;
    }
    __syncwarp();
    const int m = W.m;
    int iter = 0;
    while (!W.done) {
      if (lane == 0) {
        if (++iter > 60) {
          W.ok = 0;
          W.done = 1;
        } else {
          double g = d[l];
          double p = (d[l + 1] - g) / (2.0 * e[l]);
          double r = hypot(p, 1.0);
          if (p < 0) r = -r;
          d[l] = e[l] / (p + r);
          d[l + 1] = e[l] * (p + r);
          const double dl1 = d[l + 1];
          double h = g - d[l];
          for (int i = l + 2; i < n; ++i) d[i] -= h;
          f += h;
          p = d[m];
          double c = 1.0, c2 = c, c3 = c, s = 0.0, s2 = 0.0;
          const double el1 = e[l + 1];
          for (int i = m - 1; i >= l; --i) {
            c3 = c2;
            c2 = c;
            s2 = s;
            g = c * e[i];
            h = c * p;
            r = hypot(p, e[i]);
            e[i + 1] = s * r;
            s = e[i] / r;
            c = p / r;
            p = c * d[i] - s * g;
            d[i + 1] = h + s * (c * g + s * d[i]);
            W.cs[i] = c;
            W.sn[i] = s;
          }
          p = -s * s2 * c3 * el1 * e[l] / dl1;
          e[l] = s * p;
          d[l] = c * p;
          W.done = fabs(e[l]) > eps * tst1 ? 0 : 1;
        }
      }
      __syncwarp();
      if (!W.ok) return false;
      // the step's rotations, in the order the scalar chain made them
      if (lane < n)
        for (int i = m - 1; i >= l; --i) {
          const double c = W.cs[i], sv = W.sn[i];
          const double h = V[lane][i + 1];
          V[lane][i + 1] = sv * V[lane][i] + c * h;
          V[lane][i] = c * V[lane][i] - sv * h;
        }
      __syncwarp();
    }
    if (lane == 0) {
      d[l] += f;
      e[l] = 0.0;
    }
    __syncwarp();
  }
  if (lane == 0)
    for (int i = 0; i < n - 1; ++i) {
      int k = i;
      double p = d[i];
      for (int j = i + 1; j < n; ++j)
        if (d[j] < p) {
          k = j;
          p = d[j];
        }
      if (k != i) {
        d[k] = d[i];
        d[i] = p;
      }
      W.swaps[i] = k;
    }
  __syncwarp();
  if (lane < n)
    for (int i = 0; i < n - 1; ++i) {
      const int k = W.swaps[i];
      if (k != i) {
        const double t = V[lane][i];
        V[lane][i] = V[lane][k];
        V[lane][k] = t;
      }
    }
  __syncwarp();
  return true;
}

__device__ bool warp_symmetric_eigen(EigWork& W, int n) {
  const int lane = threadIdx.x & 31;
  double (*V)[MAXB + 1] = W.V;
  double* d = W.d;
  double* e = W.e;
  if (lane < n) d[lane] = V[n - 1][lane];
  __syncwarp();
  // tred2
  for (int i = n - 1; i > 0; --i) {
    if (lane == 0) {
      double scale = 0.0, h = 0.0;
      for (int k = 0; k < i; ++k) scale += fabs(d[k]);
      if (scale == 0.0) {
        e[i] = d[i - 1];
        for (int j = 0; j < i; ++j) {
          d[j] = V[i - 1][j];
          V[i][j] = 0.0;
          V[j][i] = 0.0;
        }
      } else {
        for (int k = 0; k < i; ++k) {
          d[k] /= scale;
          h += d[k] * d[k];
        }
        double f = d[i - 1], g = sqrt(h);
        if (f > 0) g = -g;
        e[i] = scale * g;
        h -= f * g;
        d[i - 1] = f - g;
        for (int j = 0; j < i; ++j) e[j] = 0.0;
        for (int j = 0; j < i; ++j) {
          f = d[j];
          V[j][i] = f;
          g = e[j] + V[j][j] * f;
          for (int k = j + 1; k < i; ++k) {
            g += V[k][j] * d[k];
            e[k] += V[k][j] * f;
          }
          e[j] = g;
        }
        f = 0.0;
        for (int j = 0; j < i; ++j) {
          e[j] /= h;
          f += e[j] * d[j];
        }
        const double hh = f / (h + h);
        for (int j = 0; j < i; ++j) e[j] -= hh * d[j];
      }
      W.scale = scale;
      W.h = h;
    }
    __syncwarp();
    if (W.scale != 0.0) {
      // column j of the update belongs to lane j; d[j] is refreshed once
      // every column is done (the sequential loop reads d[k], k > j, before
      // iteration k rewrites it)
      if (lane < i) {
        const double f = d[lane], g = e[lane];
        for (int k = lane; k < i; ++k) V[k][lane] -= (f * e[k] + g * d[k]);
      }
      __syncwarp();
      if (lane < i) {
        d[lane] = V[i - 1][lane];
        V[i][lane] = 0.0;
      }
      __syncwarp();
    }
    if (lane == 0) d[i] = W.h;
    __syncwarp();
  }
  for (int i = 0; i < n - 1; ++i) {
    if (lane == 0) {
      V[n - 1][i] = V[i][i];
      V[i][i] = 1.0;
    }
    __syncwarp();
    const double h = d[i + 1];
    if (h != 0.0) {
      if (lane <= i) d[lane] = V[lane][i + 1] / h;
      __syncwarp();
      if (lane <= i) {
        double g = 0.0;
        for (int k = 0; k <= i; ++k) g += V[k][i + 1] * V[k][lane];
        for (int k = 0; k <= i; ++k) V[k][lane] -= g * d[k];
      }
      __syncwarp();
    }
    if (lane <= i) V[lane][i + 1] = 0.0;
    __syncwarp();
  }
  if (lane < n) {
    d[lane] = V[n - 1][lane];
    V[n - 1][lane] = 0.0;
  }
  __syncwarp();
  if (lane == 0) {
    V[n - 1][n - 1] = 1.0;
    e[0] = 0.0;
  }
  __syncwarp();
  return warp_tql2(W, n);
}

// The projected eigenproblem of a check (eigenvector.rs:1128-1137), on the
// device: the symmetrised matrix of the steps done (its order follows from
// the step jc the host enqueued up to, or the breakdown step), its
// eigenpairs (warp_symmetric_eigen), and what the host's decisions and the
// kernels after them need: the largest eigenvalue and the residual estimate
// beta |s_last| (into st), the top Ritz vector's coefficients (svec, for
// lz_combine), and for a thick restart (eigenvector.rs:846-868) the
// coefficients of the `keep` leading Ritz vectors (srot, row-major size x p,
// for lz_rotate) and the arrowhead matrix that replaces the projected one
// (hm_next). One warp.
__global__ void __launch_bounds__(32)
lz_eigen(const double* __restrict__ hm, int m, int jc, int keep, double* __restrict__ svec,
         double* __restrict__ srot, double* __restrict__ hm_next, LzState* st) {
  __shared__ EigWork W;
  __shared__ int order[MAXB];
  const int lane = threadIdx.x;
  const int size = (st->breakdown ? st->bd_step : jc) + 1;
  for (int k = lane; k < size * size; k += 32) {
    const int r = k / size, c = k % size;
    W.V[r][c] = 0.5 * (hm[r * m + c] + hm[c * m + r]);
  }
  __syncwarp();
  if (!warp_symmetric_eigen(W, size)) {
    if (lane == 0) {
      st->eig_ok = 0;
      st->eig_size = size;
    }
    return;
  }
  int top = 0;
  for (int i = 0; i < size; ++i)
    if (W.d[i] > W.d[top]) top = i;
  const double beta = st->beta;
  if (lane < size) svec[lane] = W.V[lane][top];
  if (lane == 0) {
    st->theta_top = W.d[top];
    st->estimate = st->breakdown ? 0.0 : beta * fabs(W.V[size - 1][top]);
    st->eig_ok = 1;
    st->eig_size = size;
    // decreasing eigenvalue, ties in index order (a stable sort)
    for (int i = 0; i < size; ++i) {
      const int key = i;
      int j = i - 1;
      while (j >= 0 && W.d[order[j]] < W.d[key]) {
        order[j + 1] = order[j];
        --j;
      }
      order[j + 1] = key;
    }
  }
  __syncwarp();
  const int p = min(keep, size - 1);
  for (int l = lane; l < size; l += 32)
    for (int q = 0; q < p; ++q) srot[l * p + q] = W.V[l][order[q]];
  for (int k = lane; k < m * m; k += 32) hm_next[k] = 0.0;
  __threadfence_block();
  __syncwarp();
  if (lane < p) {
    const int q = lane;
    const double c = beta * W.V[size - 1][order[q]];
    hm_next[q * m + q] = W.d[order[q]];
    hm_next[q * m + p] = c;
    hm_next[p * m + q] = c;
  }
}

// A symmetric n x n matrix a (row-major, n <= MAXB) through the same warp
// solver: eigenvalues ascending into d, eigenvectors in the columns of V
// (row-major); *ok 0 if the QL iteration did not converge.
__global__ void __launch_bounds__(32)
small_eigen(const double* __restrict__ a, int n, double* __restrict__ d, double* __restrict__ V,
            int* ok) {
  __shared__ EigWork W;
  const int lane = threadIdx.x;
  for (int k = lane; k < n * n; k += 32) W.V[k / n][k % n] = a[k];
  __syncwarp();
  const bool good = warp_symmetric_eigen(W, n);
  if (lane == 0) *ok = good ? 1 : 0;
  if (!good) return;
  for (int k = lane; k < n; k += 32) d[k] = W.d[k];
  for (int k = lane; k < n * n; k += 32) V[k] = W.V[k / n][k % n];
}

// xx = x.x, xy = x.y, sum = sum(x); the last CTA sets value = xy / xx.
__global__ void __launch_bounds__(VB_T)
lz_dots(const double* __restrict__ x, const double* __restrict__ y, size_t dim,
        double* __restrict__ part, LzState* st) {
  double a[3] = {0, 0, 0};
  size_t r0 = (size_t)blockIdx.x * VB, r1 = min(dim, r0 + VB);
  for (size_t i = r0 + threadIdx.x; i < r1; i += VB_T) {
    double xi = x[i];
    a[0] += xi * xi;
    a[1] += xi * (y ? y[i] : 0.0);
    a[2] += xi;
  }
  block_partials<3>(a, part, 3, 3);
  if (!lz_last(&st->ticket)) return;
  if (threadIdx.x < 32) {
    double xx = fixed_block_sum(part, gridDim.x, 3, 0);
    double xy = fixed_block_sum(part, gridDim.x, 3, 1);
    double sm = fixed_block_sum(part, gridDim.x, 3, 2);
    if (threadIdx.x == 0) {
      st->xx = xx;
      st->xy = xy;
      st->sum = sm;
      st->value = xy / xx;
      st->ticket = 0;
    }
  }
}

// rinf = max |y - value x|, xinf = max |x| (eigenvector.rs:811-818).
__global__ void __launch_bounds__(VB_T)
lz_resid(const double* __restrict__ x, const double* __restrict__ y, size_t dim,
         double* __restrict__ part, LzState* st) {
  const double value = st->value;
  double r = 0, xm = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < dim;
       i += (size_t)gridDim.x * blockDim.x) {
    r = fmax(r, fabs(y[i] - value * x[i]));
    xm = fmax(xm, fabs(x[i]));
  }
  __shared__ double sh[2][VB_T / 32];
  r = warp_max(r);
  xm = warp_max(xm);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    sh[0][w] = r;
    sh[1][w] = xm;
  }
  __syncthreads();
  if (w == 0) {
    r = warp_max(lane < VB_T / 32 ? sh[0][lane] : 0.0);
    xm = warp_max(lane < VB_T / 32 ? sh[1][lane] : 0.0);
    if (lane == 0) {
      part[blockIdx.x * 2] = r;
      part[blockIdx.x * 2 + 1] = xm;
    }
  }
  if (!lz_last(&st->ticket)) return;
  if (threadIdx.x < 32) {
    const volatile double* p = part;
    double a = 0, b = 0;
    for (uint32_t q = threadIdx.x; q < gridDim.x; q += 32) {
      a = fmax(a, p[q * 2]);
      b = fmax(b, p[q * 2 + 1]);
    }
    a = warp_max(a);
    b = warp_max(b);
    if (threadIdx.x == 0) {
      st->rinf = a;
      st->xinf = b;
      st->ticket = 0;
    }
  }
}

// finish_vector (eigenvector.rs:880-899): sign by the sum, clamp negatives.
__global__ void lz_sign_clamp(double* x, size_t dim, const LzState* st) {
  const double sgn = st->sum < 0.0 ? -1.0 : 1.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < dim;
       i += (size_t)gridDim.x * blockDim.x) {
    double v = x[i] * sgn;
    x[i] = v < 0.0 ? 0.0 : v;
  }
}

// xinf = max |x| (one pass; the last CTA combines the CTA maxima).
__global__ void __launch_bounds__(VB_T)
lz_absmax(const double* __restrict__ x, size_t dim, double* __restrict__ part, LzState* st) {
  double m = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < dim;
       i += (size_t)gridDim.x * blockDim.x)
    m = fmax(m, fabs(x[i]));
  __shared__ double sh[VB_T / 32];
  m = warp_max(m);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) sh[w] = m;
  __syncthreads();
  if (w == 0) {
    m = warp_max(lane < VB_T / 32 ? sh[lane] : 0.0);
    if (lane == 0) part[blockIdx.x] = m;
  }
  if (!lz_last(&st->ticket)) return;
  if (threadIdx.x < 32) {
    const volatile double* p = part;
    double a = 0.0;
    for (uint32_t q = threadIdx.x; q < gridDim.x; q += 32) a = fmax(a, p[q]);
    a = warp_max(a);
    if (threadIdx.x == 0) {
      st->xinf = a;
      st->ticket = 0;
    }
  }
}

// x /= max |x| (how 0) or ||x|| (how 1), unless that is 0 (the scale
// option of eigenvector.rs:440-452 on non-negative scores).
__global__ void scale_by_state(double* x, size_t dim, const LzState* st, int how) {
  const double d = how == 0 ? st->xinf : sqrt(st->xx);
  if (!(d > 0.0)) return;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < dim;
       i += (size_t)gridDim.x * blockDim.x)
    x[i] = x[i] / d;
}

// x[nodes[i]] = u[i] sum(u): a component's unit vector weighted by its sum.
__global__ void scatter_by_sum(const uint32_t* __restrict__ nodes, uint32_t k,
                               const double* __restrict__ u, const LzState* st,
                               double* __restrict__ x) {
  const double f = st->sum;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < k; i += gridDim.x * blockDim.x)
    x[nodes[i]] = u[i] * f;
}

__global__ void scale_by(double* x, size_t dim, double f, int divide) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < dim;
       i += (size_t)gridDim.x * blockDim.x)
    x[i] = divide ? x[i] / f : x[i] * f;
}

__global__ void to_float(const double* __restrict__ x, size_t dim, float* __restrict__ y) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < dim;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = (float)x[i];
}

// ======================================================================= epilogues
// y_i = (A x)_i in FP64.
template <class VT>
struct PlainEpi {
  static constexpr int NACC = 0;
  double* y;
  __device__ __forceinline__ void prepare(const IterState*) {}
  static __device__ __forceinline__ void init(double*) {}
  static __device__ __forceinline__ double identity(int) { return 0.0; }
  static __device__ __forceinline__ double combine(int, double a, double b) { return a + b; }
  static __device__ __forceinline__ double warp_combine(int, double v) { return v; }
  __device__ __forceinline__ void row(uint32_t g, VT s, double*) const { y[g] = (double)s; }
  __device__ void finish(IterState*, const double*) const {}
};

// Power iteration on A' + I: y_i = (A' x)_i + x_i and the largest y.
struct PowerEpi {
  static constexpr int NACC = 1;
  const double* x;
  double* y;
  __device__ __forceinline__ void prepare(const IterState*) {}
  static __device__ __forceinline__ void init(double* a) { a[0] = 0.0; }
  static __device__ __forceinline__ double identity(int) { return 0.0; }
  static __device__ __forceinline__ double combine(int, double a, double b) { return fmax(a, b); }
  static __device__ __forceinline__ double warp_combine(int, double v) { return warp_max(v); }
  __device__ __forceinline__ void row(uint32_t g, double s, double* a) const {
    double v = s + x[g];
    y[g] = v;
    a[0] = fmax(a[0], v);
  }
  __device__ void finish(IterState* st, const double* tot) const { st->top = tot[0]; }
};

// x_new = y / top; change = max |x_new - x_old| (eigenvector.rs:341-347).
__global__ void power_vertex(const double* __restrict__ x_old, const double* __restrict__ y,
                             double* __restrict__ x_new, uint32_t n, double* __restrict__ part,
                             IterState* st) {
  if (iteration_done(st)) return;
  const double top = st->top;
  double ch = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = y[i] / top;
    x_new[i] = v;
    ch = fmax(ch, fabs(v - x_old[i]));
  }
  __shared__ double sh[VB_T / 32];
  ch = block_max(ch, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = ch;
  if (!lz_last(&st->ticket2)) return;
  if (threadIdx.x < 32) {
    const volatile double* p = part;
    double a = 0;
    for (uint32_t q = threadIdx.x; q < gridDim.x; q += 32) a = fmax(a, p[q]);
    a = warp_max(a);
    if (threadIdx.x == 0) {
      st->change = a;
      st->iter += 1;
      if (a <= st->tol) st->converged = 1;
      else if (st->iter >= st->max_iter) st->stopped = 1;
      st->ticket2 = 0;
    }
  }
}

// ======================================================================= products
// A device operator (a whole operator or a component's submatrix).
struct DevOp {
  uint32_t n = 0;
  uint64_t nnz = 0;
  const uint32_t* off = nullptr;
  const uint32_t* cols = nullptr;
  const double* v64 = nullptr;
  const float* v32 = nullptr;
  const Partition* part = nullptr;
  // owned storage for submatrices
  DevBuf<uint32_t> own_off, own_cols;
  DevBuf<double> own_v64;
  DevBuf<float> own_v32;
  std::unique_ptr<Partition> own_part;
  OpView<double> view64() const { return {n, nnz, off, cols, v64}; }
  OpView<float> view32() const { return {n, nnz, off, cols, v32}; }
};

struct SpmvScratch {
  DevBuf<double> carry64, head64, part1, part2;
  DevBuf<float> carry32, head32;
  void ensure(uint32_t ntiles) {
    if (carry64.n < ntiles + 1) {
      carry64.alloc(ntiles + 1);
      head64.alloc(ntiles + 1);
      carry32.alloc(ntiles + 1);
      head32.alloc(ntiles + 1);
      part1.alloc((size_t)ntiles * 2 + 2);
      part2.alloc(SPLIT_CTAS * 2 + 2);
    }
  }
};

constexpr int EIG_IPT = 8;
constexpr int EIG_WPB = 16;                      // warps per CTA of the product
constexpr uint32_t EIG_TILE = 32u * EIG_IPT;     // merge items per warp tile

// One product with epilogue e: merge-path warp tiles (warp_spmv) on a
// persistent grid of the CTAs that fit at once, then split_rows for the rows
// that cross tiles (and the epilogue's scalars, if any).
template <class VT, class MT, class Epi, int IPT = EIG_IPT>
static void eig_product(const OpView<MT>& v, const VT* x, const Epi& e, const Partition& P,
                        VT* carry, VT* head, double* part1, double* part2, const IterState* st,
                        cudaStream_t s) {
  constexpr size_t smem = warp_smem_bytes<VT, IPT, EIG_WPB>();
  auto fnp = warp_spmv<VT, MT, Epi, IPT, EIG_WPB, 0>;
  set_func_attr((const void*)fnp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  set_func_attr((const void*)fnp, cudaFuncAttributePreferredSharedMemoryCarveout,
                warp_fit_carveout<VT, IPT, EIG_WPB>());
  static std::mutex mu;
  static std::map<int, unsigned> cap_by_dev;  // CTAs that fit at once, per device
  int dev = 0;
  KNB_CUDA(cudaGetDevice(&dev));
  unsigned cap = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cap_by_dev.find(dev);
    if (it == cap_by_dev.end()) {
      int per_sm = 0, sms = 0;
      KNB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fnp, EIG_WPB * 32, smem));
      KNB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
      it = cap_by_dev.emplace(dev, (unsigned)std::max(1, per_sm) * (unsigned)sms).first;
    }
    cap = it->second;
  }
  const unsigned grid = std::max(1u, std::min((P.ntiles + EIG_WPB - 1) / EIG_WPB, cap));
  const uint32_t npart = std::min<uint32_t>(P.ntiles, grid * EIG_WPB);
  fnp<<<grid, EIG_WPB * 32, smem, s>>>(v, x, e, P.coords.get(), P.ntiles, carry, head, part1, st,
                                      0u);
  split_rows<VT, Epi><<<SPLIT_CTAS, SPMV_THREADS, 0, s>>>(P.split.get(), P.nsplit, P.nshort,
                                                          carry, head, e, part1, npart, part2,
                                                          const_cast<IterState*>(st));
}
// FP64 products for row shards of PageRank (shard.cu): the same warp tiles
// and split-row pass over a view whose offsets start at 0, with 4 items per
// lane (3 CTAs of 16 warps fit on an SM; 1 with 8 FP64 items), as the
// single-graph FP64 sweeps.
constexpr int SHARD_IPT = 4;
uint32_t product_tile() { return 32u * SHARD_IPT; }

void product64(const OpView<double>& v, const Partition& P, const double* x, double* y,
               ProductScratch& sc, cudaStream_t s) {
  if (sc.carry.n < (size_t)P.ntiles + 1) {
    sc.carry.alloc((size_t)P.ntiles + 1);
    sc.head.alloc((size_t)P.ntiles + 1);
    sc.part1.alloc((size_t)P.ntiles * 2 + 2);
    sc.part2.alloc(SPLIT_CTAS * 2 + 2);
  }
  PlainEpi<double> e{y};
  eig_product<double, double, PlainEpi<double>, SHARD_IPT>(
      v, x, e, P, sc.carry.get(), sc.head.get(), sc.part1.get(), sc.part2.get(), nullptr, s);
  KNB_LAUNCH("shard product");
}

// Relative residual below which FP32 products stop helping the Lanczos
// process (FP32 rounding of the products is about 1e-7 relative).
constexpr double FP32_FLOOR = 1e-5;

// y = A x (FP64 or, with x32 given, FP32 products accumulated in FP32).
static int spmv(const DevOp& A, const double* x, const float* x32, double* y, SpmvScratch& sc,
                const IterState* ist, cudaStream_t s) {
  const Partition& P = *A.part;
  sc.ensure(P.ntiles);
  if (x32) {
    PlainEpi<float> e{y};
    eig_product<float, float>(A.view32(), x32, e, P, sc.carry32.get(), sc.head32.get(),
                              sc.part1.get(), sc.part2.get(), ist, s);
  } else {
    PlainEpi<double> e{y};
    eig_product<double, double>(A.view64(), x, e, P, sc.carry64.get(), sc.head64.get(),
                                sc.part1.get(), sc.part2.get(), ist, s);
  }
  KNB_LAUNCH("spmv");
  return 2;
}

// ======================================================================= Lanczos
struct Leading {
  double value = 0;
  int64_t matvecs = 0;
  int64_t matvecs32 = 0;
};

// Thick-restart Lanczos (eigenvector.rs:746-878) on device operator A from
// the all-ones vector; the unit eigenvector is left in `xout` (device).
// Buffers of the Lanczos process, kept between calls by callers that solve
// repeatedly (they only grow).
struct LzBuffers {
  DevBuf<double> tmp, V, w, y, x, rot, hm, svec, part, srot, hm_next;
  DevBuf<float> v32;
  DevBuf<LzState> st;
  DevBuf<IterState> ist;
  SpmvScratch sc;
  LzState* hst = nullptr;
  LzBuffers() = default;
  LzBuffers(const LzBuffers&) = delete;
  LzBuffers& operator=(const LzBuffers&) = delete;
  ~LzBuffers() {
    if (hst) cudaFreeHost(hst);
  }
  template <class T>
  static void grow(DevBuf<T>& b, size_t count) {
    if (b.n < count) b.alloc(count);
  }
  void ensure(size_t dim, size_t m, bool mixed, size_t tmp_n, size_t part_n) {
    grow(tmp, tmp_n);
    grow(V, m * dim);
    grow(rot, m * dim);
    grow(w, dim);
    grow(y, dim);
    grow(x, dim);
    grow(hm, (size_t)MAXB * MAXB);
    grow(svec, (size_t)MAXB * MAXB);
    grow(srot, (size_t)MAXB * MAXB);
    grow(hm_next, (size_t)MAXB * MAXB);
    grow(part, part_n);
    if (mixed) grow(v32, dim);
    grow(st, 1);
    grow(ist, 1);
    if (!hst) KNB_CUDA(cudaMallocHost(&hst, sizeof(LzState)));
  }
};

// With B given, the operator is B A (HITS: A_b^T A_b), applied as two
// products in FP64; with `start` given (device, dim values), the process
// starts from it instead of the all-ones vector. `buf`: buffers to reuse
// (null: this call's own).
static bool symmetric_leading(const DevOp& A, double tol, double shift, int64_t max_matvecs,
                              bool mixed, double* xout, Leading* res, int* launches,
                              cudaStream_t s, const DevOp* B = nullptr,
                              const double* start = nullptr, LzBuffers* buf = nullptr,
                              bool perron = true) {
  const size_t dim = B ? B->n : A.n;
  if (B) mixed = false;
  const int m = (int)std::max<size_t>(
      1, std::min<size_t>(std::min<size_t>(dim, MAXB), std::max<size_t>((1ull << 27) / dim, 8)));
  const int keep = std::max(1, std::min(8, m >= 2 ? m - 2 : 0));
  const unsigned nb = (unsigned)((dim + VB - 1) / VB);
  const unsigned gv = grid_for(dim, 256, 148 * 16);
  LzBuffers own;
  LzBuffers& L = buf ? *buf : own;
  L.ensure(dim, (size_t)m, mixed, B ? std::max<size_t>(A.n, 1) : 0,
           std::max<size_t>((size_t)nb * (MAXB + 1), (size_t)gv * 2) + 64);
  DevBuf<double>& tmp = L.tmp;
  DevBuf<double>& V = L.V;
  DevBuf<double>& w = L.w;
  DevBuf<double>& y = L.y;
  DevBuf<double>& x = L.x;
  DevBuf<double>& rot = L.rot;
  DevBuf<float>& v32 = L.v32;
  DevBuf<double>& hm_d = L.hm;
  DevBuf<double>& svec = L.svec;
  DevBuf<double>& part = L.part;
  DevBuf<LzState>& st = L.st;
  DevBuf<IterState>& ist = L.ist;
  SpmvScratch& sc = L.sc;
  if (B) sc.ensure(std::max(A.part->ntiles, B->part->ntiles));  // no growth between products
  else sc.ensure(A.part->ntiles);
  LzState* hst = L.hst;
  auto read_state = [&] {
    KNB_CUDA(cudaMemcpyAsync(hst, st.get(), sizeof(LzState), cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
  };
  KNB_CUDA(cudaMemsetAsync(st.get(), 0, sizeof(LzState), s));
  KNB_CUDA(cudaMemsetAsync(ist.get(), 0, sizeof(IterState), s));
  KNB_CUDA(cudaMemsetAsync(hm_d.get(), 0, (size_t)m * m * 8, s));
  auto apply = [&](const double* xin, const float* x32in, double* yout,
                   const IterState* istp) -> int {
    if (!B) return spmv(A, xin, x32in, yout, sc, istp, s);
    const int l = spmv(A, xin, nullptr, tmp.get(), sc, istp, s);
    return l + spmv(*B, tmp.get(), nullptr, yout, sc, istp, s);
  };
  // v0 = start / ||start|| (blocked norm as the reference's Blocks::dot),
  // start = ones unless given
  if (start) KNB_CUDA(cudaMemcpyAsync(x.get(), start, dim * 8, cudaMemcpyDeviceToDevice, s));
  else fill_value<<<gv, 256, 0, s>>>(x.get(), (uint32_t)dim, 1.0);
  lz_dots<<<nb, VB_T, 0, s>>>(x.get(), nullptr, dim, part.get(), st.get());
  read_state();
  const double norm0 = std::sqrt(hst->xx);
  if (norm0 == 0.0 || !std::isfinite(norm0)) return false;
  scale_by<<<gv, 256, 0, s>>>(x.get(), dim, norm0, 1);
  KNB_CUDA(cudaMemcpyAsync(V.get(), x.get(), dim * 8, cudaMemcpyDeviceToDevice, s));
  if (mixed) to_float<<<gv, 256, 0, s>>>(x.get(), dim, v32.get());
  *launches += 4;

  int64_t matvecs = 0, matvecs32 = 0;
  int j0 = 0;
  bool use32 = mixed;
  double threshold = std::numeric_limits<double>::infinity();
  for (;;) {
    int j = j0;
    bool restart = false;
    while (!restart) {
      // Enqueue steps j .. jc, where jc is the next check step.
      int jc = j;
      while (!((jc + 1) == m || ((jc + 1) - j0) % 4 == 0)) ++jc;
      KNB_CUDA(cudaMemsetAsync(&ist.get()->stopped, 0, 4, s));
      int enq_from = j;
      for (int jj = j; jj <= jc; ++jj) {
        if (matvecs + (jj - enq_from) >= max_matvecs) {
          jc = jj - 1;
          break;
        }
        const double* vj = V.get() + (size_t)jj * dim;
        lz_begin<<<1, 32, 0, s>>>(st.get(), ist.get());
        *launches += 1 + apply(vj, use32 ? v32.get() : nullptr, w.get(), ist.get());
        const int cols = jj + 1, lo = cols >= 2 ? cols - 2 : 0;
        const dim3 local(nb, project_groups(cols - lo, 0)), full(nb, project_groups(cols, 1));
        lz_project<<<local, VB_T, 0, s>>>(V.get(), dim, lo, cols, w.get(), 0, part.get(), st.get(), ist.get());
        lz_subtract<<<nb, VB_T, 0, s>>>(V.get(), dim, lo, cols, w.get(), 0, part.get(), st.get(), ist.get());
        lz_project<<<full, VB_T, 0, s>>>(V.get(), dim, 0, cols, w.get(), 1, part.get(), st.get(), ist.get());
        lz_subtract<<<nb, VB_T, 0, s>>>(V.get(), dim, 0, cols, w.get(), 1, part.get(), st.get(), ist.get());
        lz_project<<<full, VB_T, 0, s>>>(V.get(), dim, 0, cols, w.get(), 2, part.get(), st.get(), ist.get());
        lz_subtract<<<nb, VB_T, 0, s>>>(V.get(), dim, 0, cols, w.get(), 2, part.get(), st.get(), ist.get());
        lz_end<<<1, 32, 0, s>>>(st.get(), ist.get(), hm_d.get(), m, jj);
        *launches += 7;
        if (jj < jc) {
          lz_next<<<gv, 256, 0, s>>>(V.get(), dim, jj + 1, w.get(), use32 ? v32.get() : nullptr,
                                     hm_d.get(), m, st.get(), ist.get(), 1);
          ++*launches;
        }
      }
      KNB_LAUNCH("lanczos step");
      if (jc < j) return false;  // matvec cap
      // The projected eigenproblem on the device; the host reads its
      // scalars with the step state, in one round trip per group of steps.
      lz_eigen<<<1, 32, 0, s>>>(hm_d.get(), m, jc, keep, svec.get(), L.srot.get(),
                                L.hm_next.get(), st.get());
      KNB_LAUNCH("lz_eigen");
      ++*launches;
      read_state();
      int jdone = hst->breakdown ? hst->bd_step : jc;
      int64_t done_now = jdone - j + 1;
      matvecs += done_now;
      if (use32) matvecs32 += done_now;
      j = jdone;
      const int size = j + 1;
      const bool breakdown = hst->breakdown != 0;
      const bool end = breakdown || size == m;
      const bool check = end || (size - j0) % 4 == 0;
      if (!check) {
        if (matvecs >= max_matvecs) return false;
        continue;  // cap reached mid-cycle; loop will return at next enqueue
      }
      if (!hst->eig_ok || hst->eig_size != size) return false;
      const double theta_top = hst->theta_top;
      const double estimate = hst->estimate;
      const double limit = tol * (std::max(theta_top, 0.0) + shift);
      if (use32 && estimate <= std::max(limit, FP32_FLOOR * (std::max(theta_top, 0.0) + shift))) {
        // FP32 products cannot resolve the residual further: restart the
        // Lanczos process with FP64 products from the current Ritz vector.
        lz_combine<<<gv, 256, 0, s>>>(V.get(), dim, size, svec.get(), x.get());
        lz_dots<<<nb, VB_T, 0, s>>>(x.get(), nullptr, dim, part.get(), st.get());
        read_state();
        KNB_CUDA(cudaMemcpyAsync(V.get(), x.get(), dim * 8, cudaMemcpyDeviceToDevice, s));
        scale_by<<<gv, 256, 0, s>>>(V.get(), dim, std::sqrt(hst->xx), 1);
        KNB_CUDA(cudaMemsetAsync(hm_d.get(), 0, (size_t)m * m * 8, s));
        KNB_CUDA(cudaMemsetAsync(st.get(), 0, sizeof(LzState), s));
        *launches += 3;
        use32 = false;
        threshold = std::numeric_limits<double>::infinity();
        j0 = 0;
        restart = true;
        continue;
      }
      if (estimate <= std::min(limit, threshold)) {
        lz_combine<<<gv, 256, 0, s>>>(V.get(), dim, size, svec.get(), x.get());
        if (matvecs >= max_matvecs) return false;
        *launches += 1 + apply(x.get(), nullptr, y.get(), nullptr);
        ++matvecs;
        lz_dots<<<nb, VB_T, 0, s>>>(x.get(), y.get(), dim, part.get(), st.get());
        lz_resid<<<gv, VB_T, 0, s>>>(x.get(), y.get(), dim, part.get(), st.get());
        *launches += 2;
        read_state();
        const double xx = hst->xx, value = hst->value, rinf = hst->rinf, xinf = hst->xinf;
        const double need = tol * (std::max(value, 0.0) + shift) * xinf;
        if (rinf <= need) {
          // finish_vector: sign, clamp, unit norm (a signed eigenvector,
          // perron false: unit norm only)
          if (perron) {
            lz_dots<<<nb, VB_T, 0, s>>>(x.get(), nullptr, dim, part.get(), st.get());
            lz_sign_clamp<<<gv, 256, 0, s>>>(x.get(), dim, st.get());
          }
          lz_dots<<<nb, VB_T, 0, s>>>(x.get(), nullptr, dim, part.get(), st.get());
          read_state();
          const double nrm = std::sqrt(hst->xx);
          if (nrm > 0.0) scale_by<<<gv, 256, 0, s>>>(x.get(), dim, nrm, 1);
          KNB_CUDA(cudaMemcpyAsync(xout, x.get(), dim * 8, cudaMemcpyDeviceToDevice, s));
          KNB_CUDA(cudaStreamSynchronize(s));
          *launches += 4;
          res->value = value;
          res->matvecs = matvecs;
          res->matvecs32 = matvecs32;
          return true;
        }
        // A failed true-residual check means FP32 products limit the
        // attainable accuracy: continue with FP64 products.
        if (use32) use32 = false;
        threshold = rinf > 0.0 ? std::min(estimate, limit) * (need / rinf) * 0.5
                               : std::min(estimate, limit) * 0.5;
        if (breakdown) {
          const double nx = std::sqrt(xx);
          KNB_CUDA(cudaMemcpyAsync(V.get(), x.get(), dim * 8, cudaMemcpyDeviceToDevice, s));
          scale_by<<<gv, 256, 0, s>>>(V.get(), dim, nx, 1);
          if (mixed) to_float<<<gv, 256, 0, s>>>(V.get(), dim, v32.get());
          KNB_CUDA(cudaMemsetAsync(hm_d.get(), 0, (size_t)m * m * 8, s));
          KNB_CUDA(cudaMemsetAsync(st.get(), 0, sizeof(LzState), s));
          *launches += 2;
          j0 = 0;
          restart = true;
          continue;
        }
      }
      if (end) {
        if (breakdown) return false;
        // thick restart from the coefficients lz_eigen left on the device
        const int p = std::min(keep, size - 1);
        lz_rotate<<<gv, 256, 0, s>>>(V.get(), dim, size, L.srot.get(), p, rot.get());
        KNB_CUDA(cudaMemcpyAsync(V.get(), rot.get(), (size_t)p * dim * 8, cudaMemcpyDeviceToDevice, s));
        KNB_CUDA(cudaMemcpyAsync(hm_d.get(), L.hm_next.get(), (size_t)m * m * 8,
                                 cudaMemcpyDeviceToDevice, s));
        KNB_CUDA(cudaMemsetAsync(&ist.get()->stopped, 0, 4, s));
        lz_next<<<gv, 256, 0, s>>>(V.get(), dim, p, w.get(), use32 ? v32.get() : nullptr,
                                   hm_d.get(), m, st.get(), ist.get(), 0);
        *launches += 2;
        j0 = p;
        restart = true;
        continue;
      }
      // continue the cycle: v = w / beta as column j + 1
      KNB_CUDA(cudaMemsetAsync(&ist.get()->stopped, 0, 4, s));
      lz_next<<<gv, 256, 0, s>>>(V.get(), dim, j + 1, w.get(), use32 ? v32.get() : nullptr,
                                 hm_d.get(), m, st.get(), ist.get(), 1);
      ++*launches;
      ++j;
    }
  }
}

// ======================================================================= HITS
static std::string fmt_g(double v);

namespace {

// The rows `nodes` of `op` with columns renumbered by `local` (device, all
// 2^32 - 1 outside the submatrix); FP64 values (1 when op has none).
void mapped_submatrix(const OpView<double>& op, const std::vector<uint32_t>& nodes,
                      const uint32_t* local, DevBuf<uint32_t>& nodes_d, DevOp& A,
                      cudaStream_t s) {
  const uint32_t kn = (uint32_t)nodes.size();
  KNB_CUDA(cudaMemcpyAsync(nodes_d.get(), nodes.data(), (size_t)kn * 4, cudaMemcpyHostToDevice,
                           s));
  A.own_off.alloc((size_t)kn + 1);
  sub_lengths_mapped<<<grid_for((uint64_t)kn * 32, 256), 256, 0, s>>>(op, nodes_d.get(), kn, local,
                                                           A.own_off.get());
  const uint64_t nnz =
      exclusive_scan<uint32_t>(A.own_off.get(), A.own_off.get(), (size_t)kn + 1, s);
  A.n = kn;
  A.nnz = nnz;
  A.own_cols.alloc(std::max<uint64_t>(nnz, 1));
  A.own_v64.alloc(std::max<uint64_t>(nnz, 1));
  sub_copy_mapped<<<grid_for((uint64_t)kn * 32, 256), 256, 0, s>>>(op, nodes_d.get(), kn, local,
                                                    A.own_off.get(), A.own_cols.get(),
                                                    A.own_v64.get());
  KNB_LAUNCH("mapped submatrix");
  A.off = A.own_off.get();
  A.cols = A.own_cols.get();
  A.v64 = A.own_v64.get();
  A.v32 = nullptr;
  A.own_part = build_partition(kn, nnz, A.off, EIG_TILE, s);
  A.part = A.own_part.get();
}

// HITS blocks (spectral.rs:757-813) on the device: every positive entry
// (i, j) of A joins hub i and authority n + j (one warp per row, the CAS
// union of the components above) and marks both as present.
__global__ void hits_union(OpView<double> a, uint32_t* parent, uint8_t* has_out, uint8_t* has_in,
                           unsigned int* any) {
  const int lane = threadIdx.x & 31;
  const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
  bool found = false;
  for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < a.n; i += warps) {
    for (uint32_t k = a.off[i] + lane; k < a.off[i + 1]; k += 32) {
      const double v = a.vals ? a.vals[k] : 1.0;
      if (!(v > 0.0)) continue;
      const uint32_t j = a.cols[k];
      found = true;
      if (!has_out[i]) has_out[i] = 1;
      if (!has_in[j]) has_in[j] = 1;
      uint32_t x = uf_find(parent, i), y = uf_find(parent, a.n + j);
      while (x != y) {
        const uint32_t lo = x < y ? x : y, hi = x < y ? y : x;
        const uint32_t old = atomicCAS(&parent[hi], hi, lo);
        if (old == hi) break;
        x = uf_find(parent, old);
        y = uf_find(parent, lo);
      }
    }
  }
  if (__any_sync(0xffffffffu, found) && lane == 0) *any = 1u;
}

// root[v] of every present node (hubs v < n with a positive entry in their
// row, authorities n + j with one in column j; the others NONE), and the
// flags of the roots. A block's root is its smallest node, so numbering the
// roots in order numbers the blocks by first appearance.
__global__ void hits_roots(uint32_t* parent, uint32_t n, const uint8_t* __restrict__ has_out,
                           const uint8_t* __restrict__ has_in, uint32_t* __restrict__ root,
                           uint32_t* __restrict__ is_root) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < 2 * n; v += gridDim.x * blockDim.x) {
    const bool present = v < n ? has_out[v] != 0 : has_in[v - n] != 0;
    const uint32_t r = present ? uf_find(parent, v) : 0xFFFFFFFFu;
    root[v] = r;
    is_root[v] = present && r == v;
  }
}

__global__ void hits_label(const uint32_t* __restrict__ root, const uint32_t* __restrict__ rank,
                           uint32_t n2, uint32_t* __restrict__ label) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n2; v += gridDim.x * blockDim.x)
    label[v] = root[v] == 0xFFFFFFFFu ? 0xFFFFFFFFu : rank[root[v]];
}

// The bounds' per-node sums (spectral.rs:814-836), one thread per row in
// CSR order: row sums of A; column sums of A and the squares of its merged
// column entries (runs of one row within a row of the transpose).
__global__ void hits_row_sum(OpView<double> a, double* __restrict__ row_sum) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    double t = 0.0;
    for (uint32_t k = a.off[i]; k < a.off[i + 1]; ++k) t = __dadd_rn(t, a.vals ? a.vals[k] : 1.0);
    row_sum[i] = t;
  }
}

__global__ void hits_col_sums(OpView<double> at, double* __restrict__ col_sum,
                              double* __restrict__ col_sq) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < at.n; j += gridDim.x * blockDim.x) {
    double sum = 0.0, q = 0.0, acc = 0.0;
    bool open = false;
    uint32_t c = 0;
    for (uint32_t k = at.off[j]; k < at.off[j + 1]; ++k) {
      const double v = at.vals ? at.vals[k] : 1.0;
      sum = __dadd_rn(sum, v);
      if (open && at.cols[k] == c) {
        acc = __dadd_rn(acc, v);
      } else {
        if (open) q = __dadd_rn(q, __dmul_rn(acc, acc));
        c = at.cols[k];
        acc = v;
        open = true;
      }
    }
    if (open) q = __dadd_rn(q, __dmul_rn(acc, acc));
    col_sum[j] = sum;
    col_sq[j] = q;
  }
}


void hits_rescale(std::vector<double>& x, int how) {
  for (double& v : x)
    if (v < 0.0) v = 0.0;
  double d = 0.0;
  if (how == 0) {
    for (double v : x) d = std::max(d, v);
  } else if (how == 1) {
    for (double v : x) d += v;
  } else {
    for (double v : x) d += v * v;
    d = std::sqrt(d);
  }
  if (d > 0.0)
    for (double& v : x) v /= d;
}

}  // namespace

// What hubs and authorities on one operator can reuse: the blocks, their
// upper bounds and order, each solved block's submatrices A_b and A_b^T with
// Kleinberg's start vector A_b^T 1, and the Lanczos buffers. Held for the
// length of a call, so concurrent calls on one operator take turns.
struct HitsPlan : Workspace {
  std::mutex mu;
  bool ready = false, any = false;
  std::vector<std::vector<uint32_t>> bh, ba;
  std::vector<double> upper;
  std::vector<size_t> order;
  struct Block {
    DevOp ab, abt;
    DevBuf<double> sdev;
    std::vector<double> sv;
  };
  std::map<size_t, std::unique_ptr<Block>> blocks;
  DevBuf<uint32_t> hub_index, auth_index, nodes_h, nodes_a;
  DevBuf<double> vdev;
  LzBuffers lz;
};

// The blocks, their bounds and their order (spectral.rs:757-836), computed
// once per operator.
static void hits_prepare(HitsPlan& plan, const OpView<double>& a64, const OpView<double>& t64,
                         uint32_t n, cudaStream_t s) {
  const uint32_t n2 = 2 * n;
  // blocks of the bipartite graph (hubs 0..n, authorities n..2n) joined by
  // positive entries (spectral.rs:757-813), found on the device
  std::vector<uint32_t> label(n2);
  unsigned int any = 0;
  {
    DevBuf<uint32_t> parent(n2), root(n2), flag((size_t)n2 + 1), lab(n2);
    DevBuf<uint8_t> has_out(n), has_in(n);
    DevBuf<unsigned int> anyd(1);
    uf_init<<<grid_for(n2, ET), ET, 0, s>>>(parent.get(), n2);
    KNB_CUDA(cudaMemsetAsync(has_out.get(), 0, n, s));
    KNB_CUDA(cudaMemsetAsync(has_in.get(), 0, n, s));
    KNB_CUDA(cudaMemsetAsync(anyd.get(), 0, 4, s));
    hits_union<<<grid_for((uint64_t)n * 32, 256), 256, 0, s>>>(a64, parent.get(), has_out.get(),
                                                               has_in.get(), anyd.get());
    hits_roots<<<grid_for(n2, ET), ET, 0, s>>>(parent.get(), n, has_out.get(), has_in.get(),
                                               root.get(), flag.get());
    KNB_LAUNCH("hub and authority blocks");
    exclusive_scan<uint32_t>(flag.get(), flag.get(), n2, s);
    hits_label<<<grid_for(n2, ET), ET, 0, s>>>(root.get(), flag.get(), n2, lab.get());
    KNB_LAUNCH("hits_label");
    KNB_CUDA(cudaMemcpyAsync(label.data(), lab.get(), (size_t)n2 * 4, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaMemcpyAsync(&any, anyd.get(), 4, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
  }
  plan.any = any != 0;
  if (!plan.any) {
    plan.ready = true;
    return;
  }
  std::vector<std::vector<uint32_t>>& bh = plan.bh;
  std::vector<std::vector<uint32_t>>& ba = plan.ba;
  for (uint32_t v = 0; v < n2; ++v) {
    const uint32_t b = label[v];
    if (b == 0xFFFFFFFFu) continue;
    if (b >= bh.size()) {
      bh.resize((size_t)b + 1);
      ba.resize((size_t)b + 1);
    }
    (v < n ? bh : ba)[b].push_back(v < n ? v : v - n);
  }
  // bounds on each block's sigma^2 (spectral.rs:814-836)
  std::vector<double> row_sum(n), col_sum(n), col_sq(n);
  {
    DevBuf<double> rs(n), cs(n), cq(n);
    hits_row_sum<<<grid_for(n, 128), 128, 0, s>>>(a64, rs.get());
    hits_col_sums<<<grid_for(n, 128), 128, 0, s>>>(t64, cs.get(), cq.get());
    KNB_LAUNCH("hub and authority bounds");
    KNB_CUDA(cudaMemcpyAsync(row_sum.data(), rs.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaMemcpyAsync(col_sum.data(), cs.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaMemcpyAsync(col_sq.data(), cq.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
  }
  const size_t kb = bh.size();
  std::vector<double>& upper = plan.upper;
  upper.assign(kb, 0.0);
  std::vector<double> lower(kb, 0.0);
  for (size_t b = 0; b < kb; ++b) {
    double rm = 0.0, cm = 0.0, lm = 0.0;
    for (uint32_t i : bh[b]) rm = std::max(rm, row_sum[i]);
    for (uint32_t j : ba[b]) {
      cm = std::max(cm, col_sum[j]);
      lm = std::max(lm, col_sq[j]);
    }
    upper[b] = rm * cm;
    lower[b] = lm;
  }
  std::vector<size_t>& order = plan.order;
  order.resize(kb);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return lower[x] > lower[y]; });
  plan.hub_index.alloc(n);
  plan.auth_index.alloc(n);
  plan.nodes_h.alloc(n);
  plan.nodes_a.alloc(n);
  KNB_CUDA(cudaMemsetAsync(plan.hub_index.get(), 0xFF, (size_t)n * 4, s));
  KNB_CUDA(cudaMemsetAsync(plan.auth_index.get(), 0xFF, (size_t)n * 4, s));
  plan.ready = true;
}

void hits(GraphHandleImpl& g, const HitsParams& p, double* hubs_out, double* auth_out,
          double* value, int* unique, cudaStream_t s) {
  const uint32_t n = g.n;
  // A: rows are arcs out of each node (matrix(g, Out, ...)); A^T: the in-CSR
  // of a directed graph (the reference's stable transpose has the same
  // entry order), A itself for an undirected one.
  const bool hdir = g.directed;
  const double lf = p.loops == 2 ? 0.0 : (!hdir && p.loops == 0 ? 2.0 : 1.0);
  Operator& A = g.op(0, p.weighted, lf, s);
  Operator& At = hdir ? g.op(1, p.weighted, lf, s) : A;
  const OpView<double> a64{A.n, A.nnz, A.rows->off.get(), A.rows->tgt.get(),
                           A.has_vals ? A.vals64.get() : nullptr};
  const OpView<double> t64{At.n, At.nnz, At.rows->off.get(), At.rows->tgt.get(),
                           At.has_vals ? At.vals64.get() : nullptr};
  HitsPlan* planp = nullptr;
  {
    std::lock_guard<std::mutex> lock(A.mu);
    if (!A.hits_ws) A.hits_ws = std::make_unique<HitsPlan>();
    planp = static_cast<HitsPlan*>(A.hits_ws.get());
  }
  HitsPlan& plan = *planp;
  std::lock_guard<std::mutex> plan_lock(plan.mu);
  if (!plan.ready) hits_prepare(plan, a64, t64, n, s);
  if (!plan.any) {
    for (uint32_t i = 0; i < n; ++i) hubs_out[i] = auth_out[i] = std::nan("");
    *value = 0.0;
    *unique = 0;
    return;
  }
  const std::vector<std::vector<uint32_t>>& bh = plan.bh;
  const std::vector<std::vector<uint32_t>>& ba = plan.ba;
  const std::vector<double>& upper = plan.upper;
  // leading eigenpair of each block that may hold the largest value
  const double TIE = 1e-9;
  double best = 0.0;
  struct Solved {
    size_t b;
    double value;
    std::vector<double> v;
    const std::vector<double>* sv;
  };
  std::vector<Solved> solved;
  int launches = 0;
  for (size_t b : plan.order) {
    if (upper[b] < best * (1.0 - TIE)) continue;
    const uint32_t nh = (uint32_t)bh[b].size(), na = (uint32_t)ba[b].size();
    std::unique_ptr<HitsPlan::Block>& blk = plan.blocks[b];
    if (!blk) {
      blk = std::make_unique<HitsPlan::Block>();
      DevBuf<uint32_t>& nodes_h = plan.nodes_h;
      DevBuf<uint32_t>& nodes_a = plan.nodes_a;
      KNB_CUDA(cudaMemcpyAsync(nodes_h.get(), bh[b].data(), (size_t)nh * 4, cudaMemcpyHostToDevice, s));
      KNB_CUDA(cudaMemcpyAsync(nodes_a.get(), ba[b].data(), (size_t)na * 4, cudaMemcpyHostToDevice, s));
      scatter_local<<<grid_for(nh, 256), 256, 0, s>>>(nodes_h.get(), nh, plan.hub_index.get());
      scatter_local<<<grid_for(na, 256), 256, 0, s>>>(nodes_a.get(), na, plan.auth_index.get());
      DevBuf<uint32_t> tmp_nodes(std::max(nh, na));
      mapped_submatrix(a64, bh[b], plan.auth_index.get(), tmp_nodes, blk->ab, s);
      mapped_submatrix(t64, ba[b], plan.hub_index.get(), tmp_nodes, blk->abt, s);
      unscatter_local<<<grid_for(nh, 256), 256, 0, s>>>(nodes_h.get(), nh, plan.hub_index.get());
      unscatter_local<<<grid_for(na, 256), 256, 0, s>>>(nodes_a.get(), na, plan.auth_index.get());
      // Kleinberg's first authority vector A_b^T 1
      DevBuf<double> ones(std::max<uint32_t>(nh, 1));
      blk->sdev.alloc(std::max<uint32_t>(na, 1));
      fill_value<<<grid_for(nh, 256), 256, 0, s>>>(ones.get(), nh, 1.0);
      SpmvScratch sc;
      launches += 6 + spmv(blk->abt, ones.get(), nullptr, blk->sdev.get(), sc, nullptr, s);
      blk->sv.resize(na);
      KNB_CUDA(cudaMemcpyAsync(blk->sv.data(), blk->sdev.get(), (size_t)na * 8,
                               cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaStreamSynchronize(s));
    }
    if (plan.vdev.n < na) plan.vdev.alloc(na);
    Leading res;
    if (!symmetric_leading(blk->ab, p.tol, 0.0, p.max_iter, false, plan.vdev.get(), &res,
                           &launches, s, &blk->abt, blk->sdev.get(), &plan.lz))
      throw Error("hub and authority scores did not converge to tolerance " + fmt_g(p.tol) +
                  " within " + std::to_string(p.max_iter) +
                  " matrix-vector products; a larger iteration cap may help");
    Solved sol;
    sol.b = b;
    sol.value = res.value;
    sol.v.resize(na);
    sol.sv = &blk->sv;
    KNB_CUDA(cudaMemcpyAsync(sol.v.data(), plan.vdev.get(), (size_t)na * 8, cudaMemcpyDeviceToHost,
                             s));
    KNB_CUDA(cudaStreamSynchronize(s));
    best = std::max(best, res.value);
    solved.push_back(std::move(sol));
  }
  std::vector<double> auth(n, 0.0);
  int tied = 0;
  for (const Solved& sol : solved) {
    if (sol.value < best * (1.0 - TIE)) continue;
    ++tied;
    double weight = 0.0;
    for (size_t i = 0; i < sol.v.size(); ++i) weight += sol.v[i] * (*sol.sv)[i];
    for (size_t i = 0; i < ba[sol.b].size(); ++i) auth[ba[sol.b][i]] = sol.v[i] * weight;
  }
  // hubs = A auth (device product)
  DevBuf<double> ad(n), hd(n);
  KNB_CUDA(cudaMemcpyAsync(ad.get(), auth.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
  DevOp full;
  full.n = A.n;
  full.nnz = A.nnz;
  full.off = A.rows->off.get();
  full.cols = A.rows->tgt.get();
  full.v64 = A.has_vals ? A.vals64.get() : nullptr;
  full.part = &A.partition(EIG_TILE, s);
  SpmvScratch sc;
  spmv(full, ad.get(), nullptr, hd.get(), sc, nullptr, s);
  std::vector<double> hubs(n);
  KNB_CUDA(cudaMemcpyAsync(hubs.data(), hd.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  hits_rescale(auth, p.scale);
  hits_rescale(hubs, p.scale);
  memcpy(hubs_out, hubs.data(), (size_t)n * 8);
  memcpy(auth_out, auth.data(), (size_t)n * 8);
  *value = best;
  *unique = tied == 1 ? 1 : 0;
}

// ======================================================================= driver
static std::string fmt_g(double v) {
  char b[64];
  snprintf(b, sizeof b, "%g", v);
  return b;
}

static void scale_host(std::vector<double>& x, int how) {
  double d = 0.0;
  if (how == 0) {
    for (double v : x) d = std::max(d, v);
  } else {
    for (double v : x) d += v * v;
    d = std::sqrt(d);
  }
  if (d > 0.0)
    for (double& v : x) v /= d;
}

// What an eigenvector solve on one operator can reuse: its components and
// whether any of them is cyclic; for symmetric operators the per-component
// bounds and order, the submatrices of the components solved so far (with
// their partitions), and the Lanczos buffers. Held for the length of a
// solve, so concurrent solves on one operator take turns.
struct EigPlan : Workspace {
  std::mutex mu;
  bool ready = false;
  Comps comps;
  unsigned int cyclic = 0;
  bool sym_ready = false;
  std::vector<double> upper, lower;
  std::vector<size_t> order, start;
  std::vector<uint32_t> members;
  std::map<size_t, std::unique_ptr<DevOp>> subs;
  std::map<size_t, DevBuf<double>> vecs;  // each solved component's unit vector
  DevBuf<uint32_t> local, members_d;
  DevBuf<double> xd;
  LzBuffers lz;
};

void eigenvector(GraphHandleImpl& g, const EigenParams& p, double* out, EigenResult* r,
                 cudaStream_t s) {
  const uint32_t n = g.n;
  if (n == 0) {
    r->eigenvalue = std::numeric_limits<double>::quiet_NaN();
    r->connected = true;
    return;
  }
  cudaEvent_t t0, t1;
  KNB_CUDA(cudaEventCreate(&t0));
  KNB_CUDA(cudaEventCreate(&t1));
  KNB_CUDA(cudaEventRecord(t0, s));
  int launches = 0;
  const int mode = g.directed ? p.mode : 3;
  const bool hdir = g.directed && mode != 3;
  const int which = !g.directed ? 0 : (mode == 3 ? 2 : (mode == 2 ? 1 : 0));
  const double lf = p.loops == 2 ? 0.0 : (!hdir && p.loops == 0 ? 2.0 : 1.0);
  Operator& op = g.op(which, p.weighted, lf, s);
  const unsigned gv = grid_for(n, 256, 148 * 16);
  EigPlan* planp = nullptr;
  {
    std::lock_guard<std::mutex> lock(op.mu);
    if (!op.eig_ws) op.eig_ws = std::make_unique<EigPlan>();
    planp = static_cast<EigPlan*>(op.eig_ws.get());
  }
  EigPlan& plan = *planp;
  std::lock_guard<std::mutex> plan_lock(plan.mu);
  OpView<double> v64 = op.view64();

  // components: strong (directed h) or weak; whether any is cyclic
  if (!plan.ready) {
    if (hdir) {
      plan.comps = strong_components(g, nullptr, false, &launches, s);
    } else {
      plan.comps = weak_components(g, s);
      launches += 5;
    }
    DevBuf<uint32_t> comp(n);
    DevBuf<unsigned int> flag(1);
    KNB_CUDA(cudaMemcpyAsync(comp.get(), plan.comps.membership.data(), (size_t)n * 4,
                             cudaMemcpyHostToDevice, s));
    KNB_CUDA(cudaMemsetAsync(flag.get(), 0, 4, s));
    cyclic_arcs<<<grid_for(n, 256), 256, 0, s>>>(v64, comp.get(), flag.get());
    ++launches;
    KNB_CUDA(cudaMemcpyAsync(&plan.cyclic, flag.get(), 4, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    plan.ready = true;
  }
  const Comps& strong = plan.comps;
  r->connected = strong.count() == 1;
  const unsigned int cyc = plan.cyclic;
  if (plan.xd.n < n) plan.xd.alloc(n);
  DevBuf<double>& xd = plan.xd;
  if (!cyc) {
    std::vector<double> x(n);
    fill_value<<<gv, 256, 0, s>>>(xd.get(), n, 1.0);
    sink_scores<<<grid_for(n, 256), 256, 0, s>>>(v64, xd.get());
    launches += 2;
    KNB_CUDA(cudaMemcpyAsync(x.data(), xd.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    scale_host(x, p.scale);
    memcpy(out, x.data(), (size_t)n * 8);
    r->eigenvalue = 0.0;
    r->matvecs = 0;
  } else if (hdir) {
    // power iteration on A' + I (eigenvector.rs:330-374)
    const Partition& P = op.partition(EIG_TILE, s);
    DevBuf<double> xb[2] = {DevBuf<double>(n), DevBuf<double>(n)}, y(n);
    DevBuf<double> carry(P.ntiles + 1), head(P.ntiles + 1), part1((size_t)P.ntiles + 2),
        part2(SPLIT_CTAS + 2), part3(gv + 2);
    DevBuf<IterState> st(1);
    IterState is{};
    is.tol = p.tol;
    is.max_iter = (int32_t)std::min<int64_t>(p.max_iter, INT32_MAX);
    KNB_CUDA(cudaMemcpyAsync(st.get(), &is, sizeof(is), cudaMemcpyHostToDevice, s));
    fill_value<<<gv, 256, 0, s>>>(xb[0].get(), n, 1.0);
    ++launches;
    IterState hs{};
    int batch = 0;
    for (;;) {
      for (int k = 0; k < 8; ++k) {
        int b = k & 1;
        PowerEpi e{xb[b].get(), y.get()};
        eig_product<double, double>(v64, xb[b].get(), e, P, carry.get(), head.get(), part1.get(),
                                    part2.get(), st.get(), s);
        power_vertex<<<gv, 256, 0, s>>>(xb[b].get(), y.get(), xb[1 - b].get(), n, part3.get(), st.get());
        launches += 3;
      }
      KNB_LAUNCH("power iteration");
      KNB_CUDA(cudaMemcpyAsync(&hs, st.get(), sizeof(hs), cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaStreamSynchronize(s));
      ++batch;
      if (hs.converged || hs.stopped) break;
    }
    if (!hs.converged)
      throw Error("eigenvector centrality did not converge to tolerance " + fmt_g(p.tol) +
                  " within " + std::to_string(p.max_iter) +
                  " iterations. Power iteration converges slowly when the largest eigenvalue is "
                  "close to the next one, and not at all to a single answer when several "
                  "strongly connected components share it; a larger iteration cap may help in "
                  "the first case");
    double* xf = xb[hs.iter & 1].get();
    // eigenvalue sum(A'x) / sum(x), scores times sum(x) / sum(x^2)
    DevOp A;
    A.n = n;
    A.nnz = op.nnz;
    A.off = op.rows->off.get();
    A.cols = op.rows->tgt.get();
    A.v64 = op.has_vals ? op.vals64.get() : nullptr;
    A.part = &P;
    SpmvScratch sc;
    launches += spmv(A, xf, nullptr, y.get(), sc, nullptr, s);
    std::vector<double> hx(n), hy(n);
    KNB_CUDA(cudaMemcpyAsync(hx.data(), xf, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaMemcpyAsync(hy.data(), y.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    double s0 = 0, s1 = 0, s2 = 0;
    for (uint32_t v = 0; v < n; ++v) {
      s0 += hy[v];
      s1 += hx[v];
      s2 += hx[v] * hx[v];
    }
    r->eigenvalue = s1 > 0.0 ? s0 / s1 : 0.0;
    if (s2 > 0.0) {
      double wgt = s1 / s2;
      for (double& xv : hx) xv *= wgt;
    }
    r->matvecs = hs.iter;
    scale_host(hx, p.scale);
    memcpy(out, hx.data(), (size_t)n * 8);
  } else {
    // symmetric: Lanczos per weak component (eigenvector.rs:383-479)
    const Comps& comps = strong;  // weak components of h
    const size_t k = comps.count();
    if (!plan.sym_ready) {
      DevBuf<double> sdev(n), qdev(n);
      op_row_sums<<<grid_for((uint64_t)n * 32, 256), 256, 0, s>>>(v64, sdev.get(), qdev.get());
      ++launches;
      std::vector<double> rs(n), rq(n);
      KNB_CUDA(cudaMemcpyAsync(rs.data(), sdev.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaMemcpyAsync(rq.data(), qdev.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaStreamSynchronize(s));
      std::vector<double> sum(k, 0.0), square(k, 0.0);
      plan.upper.assign(k, 0.0);
      plan.lower.assign(k, 0.0);
      for (uint32_t v = 0; v < n; ++v) {
        uint32_t c = comps.membership[v];
        plan.upper[c] = std::max(plan.upper[c], rs[v]);
        sum[c] += rs[v];
        square[c] = std::max(square[c], rq[v]);
      }
      for (size_t c = 0; c < k; ++c)
        plan.lower[c] = std::max(sum[c] / (double)comps.sizes[c], std::sqrt(square[c]));
      plan.order.resize(k);
      std::iota(plan.order.begin(), plan.order.end(), 0);
      std::stable_sort(plan.order.begin(), plan.order.end(),
                       [&](size_t a, size_t b) { return plan.lower[b] < plan.lower[a]; });
      plan.start.assign(k + 1, 0);
      for (uint32_t c : comps.membership) plan.start[c + 1]++;
      for (size_t c = 0; c < k; ++c) plan.start[c + 1] += plan.start[c];
      plan.members.resize(n);
      std::vector<size_t> cur(plan.start.begin(), plan.start.end() - 1);
      for (uint32_t v = 0; v < n; ++v) plan.members[cur[comps.membership[v]]++] = v;
      plan.members_d.alloc(n);
      KNB_CUDA(cudaMemcpyAsync(plan.members_d.get(), plan.members.data(), (size_t)n * 4,
                               cudaMemcpyHostToDevice, s));
      if (k > 1) plan.local.alloc(n);
      plan.sym_ready = true;
    }
    const std::vector<double>& upper = plan.upper;
    const std::vector<size_t>& order = plan.order;
    const std::vector<size_t>& start = plan.start;
    double best = 0.0;
    int64_t matvecs = 0, matvecs32 = 0;
    struct Solved {
      size_t c;
      double value;
      double* u;
    };
    std::vector<Solved> solved;
    DevBuf<uint32_t>& local = plan.local;
    const double TIE = 1e-9;
    for (size_t c : order) {
      if (upper[c] <= 0.0 || upper[c] < best * (1.0 - TIE)) continue;
      const uint32_t kn = (uint32_t)(start[c + 1] - start[c]);
      DevOp whole;
      std::unique_ptr<DevOp>& cached = plan.subs[c];
      const bool build_sub = k != 1 && !cached;
      if (build_sub) cached = std::make_unique<DevOp>();
      DevOp& A = k == 1 ? whole : *cached;
      if (k == 1) {
        A.n = n;
        A.nnz = op.nnz;
        A.off = op.rows->off.get();
        A.cols = op.rows->tgt.get();
        A.v64 = op.has_vals ? op.vals64.get() : nullptr;
        A.v32 = op.has_vals ? op.vals32.get() : nullptr;
        A.part = &op.partition(EIG_TILE, s);
      } else if (build_sub) {
        const uint32_t* nodes_d = plan.members_d.get() + start[c];
        scatter_local<<<grid_for(kn, 256), 256, 0, s>>>(nodes_d, kn, local.get());
        A.own_off.alloc((size_t)kn + 1);
        sub_lengths<<<grid_for(kn + 1, 256), 256, 0, s>>>(op.rows->off.get(), nodes_d, kn,
                                                          A.own_off.get());
        uint64_t nnz = exclusive_scan<uint32_t>(A.own_off.get(), A.own_off.get(), (size_t)kn + 1, s);
        A.n = kn;
        A.nnz = nnz;
        A.own_cols.alloc(std::max<uint64_t>(nnz, 1));
        if (op.has_vals) {
          A.own_v64.alloc(std::max<uint64_t>(nnz, 1));
          A.own_v32.alloc(std::max<uint64_t>(nnz, 1));
        }
        sub_copy<<<grid_for((uint64_t)kn * 32, 256), 256, 0, s>>>(v64, nodes_d, kn, local.get(),
                                                   A.own_off.get(), A.own_cols.get(),
                                                   op.has_vals ? A.own_v64.get() : nullptr,
                                                   op.has_vals ? A.own_v32.get() : nullptr);
        KNB_LAUNCH("submatrix");
        launches += 4;
        A.off = A.own_off.get();
        A.cols = A.own_cols.get();
        A.v64 = op.has_vals ? A.own_v64.get() : nullptr;
        A.v32 = op.has_vals ? A.own_v32.get() : nullptr;
        A.own_part = build_partition(kn, nnz, A.off, EIG_TILE, s);
        A.part = A.own_part.get();
      }
      Solved sv;
      sv.c = c;
      DevBuf<double>& u = plan.vecs[c];
      if (u.n < kn) u.alloc(kn);
      sv.u = u.get();
      Leading res;
      if (!symmetric_leading(A, p.tol, 1.0, p.max_iter, p.precision == 1, sv.u, &res,
                             &launches, s, nullptr, nullptr, &plan.lz))
        throw Error("eigenvector centrality did not converge to tolerance " + fmt_g(p.tol) +
                    " within " + std::to_string(p.max_iter) +
                    " matrix-vector products; a larger iteration cap may help");
      matvecs += res.matvecs;
      matvecs32 += res.matvecs32;
      best = std::max(best, res.value);
      sv.value = res.value;
      solved.push_back(std::move(sv));
    }
    // tied components' vectors, each weighted by its sum, then the scale
    // option; all on the device, one copy of the scores to the host
    fill_value<<<gv, 256, 0, s>>>(xd.get(), n, 0.0);
    ++launches;
    LzBuffers::grow(plan.lz.st, 1);
    LzBuffers::grow(plan.lz.part, std::max<size_t>(gv, 3 * ((size_t)n + VB - 1) / VB) + 64);
    LzState* st = plan.lz.st.get();
    double* part = plan.lz.part.get();
    KNB_CUDA(cudaMemsetAsync(st, 0, sizeof(LzState), s));
    for (auto& sv : solved) {
      if (sv.value < best * (1.0 - TIE)) continue;
      const uint32_t kn = (uint32_t)(start[sv.c + 1] - start[sv.c]);
      lz_dots<<<(unsigned)((kn + VB - 1) / VB), VB_T, 0, s>>>(sv.u, nullptr, kn, part, st);
      scatter_by_sum<<<grid_for(kn, 256), 256, 0, s>>>(plan.members_d.get() + start[sv.c], kn,
                                                       sv.u, st, xd.get());
      launches += 2;
    }
    if (p.scale == 0)
      lz_absmax<<<gv, VB_T, 0, s>>>(xd.get(), n, part, st);
    else
      lz_dots<<<(unsigned)((n + VB - 1) / VB), VB_T, 0, s>>>(xd.get(), nullptr, n, part, st);
    scale_by_state<<<gv, 256, 0, s>>>(xd.get(), n, st, p.scale == 0 ? 0 : 1);
    launches += 2;
    KNB_LAUNCH("eigenvector scores");
    KNB_CUDA(cudaMemcpyAsync(out, xd.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    r->eigenvalue = best;
    r->matvecs = matvecs;
    r->matvecs_fp32 = matvecs32;
  }
  KNB_CUDA(cudaEventRecord(t1, s));
  KNB_CUDA(cudaEventSynchronize(t1));
  float ms = 0;
  KNB_CUDA(cudaEventElapsedTime(&ms, t0, t1));
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  r->seconds = ms * 1e-3;
  r->kernel_launches = launches;
}

// ======================================================================= leading eigenvector communities
// Newman's leading eigenvector method (crates/engine/src/metrics/partition/
// leading_eigen.rs:57-160): groups are divided by the signs of the leading
// eigenvector of their generalized modularity matrix B(g), breadth first,
// until no division has a positive eigenvalue and a positive gain.
// The dense adjacency, the degrees, B(g), its row sums and the gain are
// computed on the device in the reference's summation order (one thread per
// row, in column order); the leading eigenpair comes from the thick-restart
// Lanczos process above in FP64 on B(g) as a dense operator, without the
// Perron clamp, started from a fixed hashed vector (B(g) 1 = 0, so the
// all-ones start of eigenvector centrality would break down at once). Rows
// of B(g) that are entirely zero (nodes without ties) have eigenvector
// component exactly 0 for any eigenvalue other than 0, so they stay out of
// the eigenproblem and take component 0, as the reference's dense solver
// gives them (to rounding). The reference's scale sum runs over the whole
// matrix in one sequence; here it is the sum of the per-row sums.

// a[u n + v]: arcs of row u in CSR order (input order per target), a loop
// adding twice its weight (leading_eigen.rs:70-80).
__global__ void le_dense(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                         const double* __restrict__ w, uint32_t n, double* __restrict__ a) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    double* row = a + (size_t)u * n;
    for (uint32_t k = off[u]; k < off[u + 1]; ++k) {
      const uint32_t v = tgt[k];
      const double x = w ? w[k] : 1.0;
      if (v == u) row[u] = __dadd_rn(row[u], __dmul_rn(2.0, x));
      else row[v] = __dadd_rn(row[v], x);
    }
  }
}

__global__ void le_row_sums(const double* __restrict__ a, uint32_t n, double* __restrict__ k) {
  for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
    const double* row = a + (size_t)u * n;
    double t = 0.0;
    for (uint32_t j = 0; j < n; ++j) t = __dadd_rn(t, row[j]);
    k[u] = t;
  }
}

// b[r ng + c] = a[i n + j] - k_i k_j / 2m for group members i = g[r], j = g[c].
__global__ void le_build(const double* __restrict__ a, uint32_t n, const double* __restrict__ k,
                         double two_m, const uint32_t* __restrict__ grp, uint32_t ng,
                         double* __restrict__ b) {
  const uint64_t total = (uint64_t)ng * ng;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = (uint32_t)(q / ng), c = (uint32_t)(q % ng);
    const uint32_t i = grp[r], j = grp[c];
    b[q] = __dsub_rn(a[(size_t)i * n + j], __ddiv_rn(__dmul_rn(k[i], k[j]), two_m));
  }
}

// Per row: the diagonal minus the row's sum, then the sum of |b| over the row.
__global__ void le_diag(double* __restrict__ b, uint32_t ng, double* __restrict__ absrow) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < ng; r += gridDim.x * blockDim.x) {
    double* row = b + (size_t)r * ng;
    double t = 0.0;
    for (uint32_t c = 0; c < ng; ++c) t = __dadd_rn(t, row[c]);
    row[r] = __dsub_rn(row[r], t);
    double z = 0.0;
    for (uint32_t c = 0; c < ng; ++c) z = __dadd_rn(z, fabs(row[c]));
    absrow[r] = z;
  }
}

// The dense operator over the rows `nz` of B(g) as a CSR matrix.
__global__ void le_sub(const double* __restrict__ b, uint32_t ng, const uint32_t* __restrict__ nz,
                       uint32_t dim, uint32_t* __restrict__ off, uint32_t* __restrict__ cols,
                       double* __restrict__ vals) {
  const uint64_t total = (uint64_t)dim * dim;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t r = (uint32_t)(q / dim), c = (uint32_t)(q % dim);
    cols[q] = c;
    vals[q] = b[(size_t)nz[r] * ng + nz[c]];
    if (c == 0) off[r] = (uint32_t)q;
    if (q == 0) off[dim] = (uint32_t)total;
  }
}

// A fixed start vector with values in [-1, 1) from a hash of the index.
__global__ void le_start(double* __restrict__ x, uint32_t dim) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < dim; r += gridDim.x * blockDim.x) {
    uint64_t z = (uint64_t)r * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    x[r] = (double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  }
}

// s_r times the sum over c of b[r][c] s_c, in column order.
__global__ void le_gain_rows(const double* __restrict__ b, uint32_t ng, const double* __restrict__ sv,
                             double* __restrict__ out) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < ng; r += gridDim.x * blockDim.x) {
    const double* row = b + (size_t)r * ng;
    double t = 0.0;
    for (uint32_t c = 0; c < ng; ++c) t = __dadd_rn(t, __dmul_rn(row[c], sv[c]));
    out[r] = __dmul_rn(sv[r], t);
  }
}

void leading_eigen(GraphHandleImpl& g, bool weighted, int64_t* membership, double* q,
                   int64_t* splits_out, int* launches_out, cudaStream_t s) {
  const uint32_t n = g.n;
  int launches = 0;
  std::vector<size_t> memb(n, 0);
  size_t splits = 0;
  double two_m = 0.0;
  DevBuf<double> a, k;
  if (n > 0) {
    a.alloc((size_t)n * n);
    k.alloc(n);
    KNB_CUDA(cudaMemsetAsync(a.get(), 0, (size_t)n * n * 8, s));
    le_dense<<<grid_for(n, 128), 128, 0, s>>>(g.out.off.get(), g.out.tgt.get(),
                                                weighted ? g.out.w.get() : nullptr, n, a.get());
    le_row_sums<<<grid_for(n, 128), 128, 0, s>>>(a.get(), n, k.get());
    KNB_LAUNCH("leading eigenvector adjacency");
    launches += 2;
    std::vector<double> hk(n);
    KNB_CUDA(cudaMemcpyAsync(hk.data(), k.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    for (double v : hk) two_m += v;
  }
  if (two_m > 0.0) {
    size_t next_label = 1;
    std::deque<std::vector<uint32_t>> queue;
    {
      std::vector<uint32_t> all(n);
      std::iota(all.begin(), all.end(), 0u);
      queue.push_back(std::move(all));
    }
    DevBuf<double> b, absrow, vals, x, start, sv, rowgain;
    DevBuf<uint32_t> grp, nzd, off, cols;
    LzBuffers lz;
    while (!queue.empty()) {
      std::vector<uint32_t> group = std::move(queue.front());
      queue.pop_front();
      const uint32_t ng = (uint32_t)group.size();
      if (ng < 2) continue;
      const size_t nn = (size_t)ng * ng;
      if (b.n < nn) b.alloc(nn);
      if (grp.n < ng) {
        grp.alloc(ng);
        absrow.alloc(ng);
        sv.alloc(ng);
        rowgain.alloc(ng);
      }
      KNB_CUDA(cudaMemcpyAsync(grp.get(), group.data(), (size_t)ng * 4, cudaMemcpyHostToDevice, s));
      le_build<<<grid_for(nn, 256), 256, 0, s>>>(a.get(), n, k.get(), two_m, grp.get(), ng, b.get());
      le_diag<<<grid_for(ng, 128), 128, 0, s>>>(b.get(), ng, absrow.get());
      KNB_LAUNCH("generalized modularity matrix");
      launches += 2;
      std::vector<double> habs(ng);
      KNB_CUDA(cudaMemcpyAsync(habs.data(), absrow.get(), (size_t)ng * 8, cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaStreamSynchronize(s));
      double total = 0.0, maxrow = 0.0;
      std::vector<uint32_t> nz;
      for (uint32_t r = 0; r < ng; ++r) {
        total += habs[r];
        maxrow = std::max(maxrow, habs[r]);
        if (habs[r] > 0.0) nz.push_back(r);
      }
      const double scale = total / (double)ng;
      // leading eigenpair of B(g) over its nonzero rows
      double lambda = 0.0;
      std::vector<double> u(ng, 0.0);
      if (!nz.empty()) {
        const uint32_t dim = (uint32_t)nz.size();
        const size_t nnz = (size_t)dim * dim;
        if (nnz > 0xFFFFFFFFull) throw Error("group too large for the leading eigenvector method");
        if (vals.n < nnz) {
          vals.alloc(nnz);
          cols.alloc(nnz);
        }
        if (off.n < (size_t)dim + 1) {
          off.alloc((size_t)dim + 1);
          nzd.alloc(dim);
          x.alloc(dim);
          start.alloc(dim);
        }
        KNB_CUDA(cudaMemcpyAsync(nzd.get(), nz.data(), (size_t)dim * 4, cudaMemcpyHostToDevice, s));
        le_sub<<<grid_for(nnz, 256), 256, 0, s>>>(b.get(), ng, nzd.get(), dim, off.get(), cols.get(),
                                                  vals.get());
        le_start<<<grid_for(dim, 256), 256, 0, s>>>(start.get(), dim);
        KNB_LAUNCH("modularity operator");
        launches += 2;
        DevOp A;
        A.n = dim;
        A.nnz = nnz;
        A.off = off.get();
        A.cols = cols.get();
        A.v64 = vals.get();
        A.own_part = build_partition(dim, nnz, A.off, EIG_TILE, s);
        A.part = A.own_part.get();
        Leading res;
        if (!symmetric_leading(A, 1e-12, maxrow, 200000, false, x.get(), &res, &launches, s,
                               nullptr, start.get(), &lz, false))
          throw Error("the leading eigenvector method: the eigenvector of a group of " +
                      std::to_string(ng) + " nodes did not converge");
        lambda = res.value;
        std::vector<double> hx(dim);
        KNB_CUDA(cudaMemcpyAsync(hx.data(), x.get(), (size_t)dim * 8, cudaMemcpyDeviceToHost, s));
        KNB_CUDA(cudaStreamSynchronize(s));
        for (uint32_t r = 0; r < dim; ++r) u[nz[r]] = hx[r];
      }
      if (std::isnan(lambda) || lambda <= 1e-10 * scale) continue;
      // the first component of largest magnitude decides the sign
      uint32_t big = 0;
      for (uint32_t r = 1; r < ng; ++r)
        if (std::fabs(u[r]) > std::fabs(u[big])) big = r;
      const double sign = u[big] < 0.0 ? -1.0 : 1.0;
      const double tiny = 1e-12 * std::fabs(u[big]);
      std::vector<double> sg(ng);
      for (uint32_t r = 0; r < ng; ++r) sg[r] = sign * u[r] > tiny ? 1.0 : -1.0;
      KNB_CUDA(cudaMemcpyAsync(sv.get(), sg.data(), (size_t)ng * 8, cudaMemcpyHostToDevice, s));
      le_gain_rows<<<grid_for(ng, 128), 128, 0, s>>>(b.get(), ng, sv.get(), rowgain.get());
      KNB_LAUNCH("modularity gain");
      ++launches;
      std::vector<double> hg(ng);
      KNB_CUDA(cudaMemcpyAsync(hg.data(), rowgain.get(), (size_t)ng * 8, cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaStreamSynchronize(s));
      double gain = 0.0;
      for (double v : hg) gain += v;
      if (std::isnan(gain) || gain <= 1e-10 * scale * (double)ng) continue;
      std::vector<uint32_t> plus, minus;
      for (uint32_t r = 0; r < ng; ++r) (sg[r] > 0.0 ? plus : minus).push_back(group[r]);
      if (plus.empty() || minus.empty()) continue;
      for (uint32_t v : minus) memb[v] = next_label;
      ++next_label;
      ++splits;
      queue.push_back(std::move(plus));
      queue.push_back(std::move(minus));
    }
  } else {
    std::iota(memb.begin(), memb.end(), (size_t)0);
  }
  // labels by first appearance (partition.rs:62-65)
  std::unordered_map<size_t, int64_t> seen;
  std::vector<int64_t> label(n);
  for (uint32_t v = 0; v < n; ++v) {
    auto it = seen.find(memb[v]);
    if (it == seen.end()) it = seen.emplace(memb[v], (int64_t)seen.size()).first;
    label[v] = it->second;
  }
  // modularity of the partition on the input network
  // (crates/engine/src/metrics/community.rs:97-146, undirected, resolution 1)
  const size_t kc = seen.size();
  std::vector<double> inside(kc, 0.0), kout(kc, 0.0), kin(kc, 0.0);
  double m = 0.0;
  if (g.m) {
    std::vector<uint32_t> hs(g.m), ht(g.m);
    std::vector<double> hw(weighted ? g.m : 0);
    KNB_CUDA(cudaMemcpyAsync(hs.data(), g.src.get(), g.m * 4, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaMemcpyAsync(ht.data(), g.tgt.get(), g.m * 4, cudaMemcpyDeviceToHost, s));
    if (weighted) KNB_CUDA(cudaMemcpyAsync(hw.data(), g.w.get(), g.m * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    for (uint64_t e = 0; e < g.m; ++e) {
      const double xv = weighted ? hw[e] : 1.0;
      const int64_t cs = label[hs[e]], ct = label[ht[e]];
      m += xv;
      kout[cs] += xv;
      kin[ct] += xv;
      if (cs == ct) inside[cs] += xv;
    }
  }
  double qv = std::numeric_limits<double>::quiet_NaN();
  if (m > 0.0) {
    qv = 0.0;
    for (size_t c = 0; c < kc; ++c) {
      const double kk = kout[c] + kin[c];
      qv += inside[c] / m - (kk / (2.0 * m)) * (kk / (2.0 * m));
    }
  }
  for (uint32_t v = 0; v < n; ++v) membership[v] = label[v];
  *q = qv;
  *splits_out = (int64_t)splits;
  if (launches_out) *launches_out = launches;
}

bool symmetric_eigen_device(const double* a, int n, double* d, double* V, cudaStream_t s) {
  if (n < 0 || n > MAXB) throw Error("the projected eigensolver takes matrices of order 0.." +
                                     std::to_string(MAXB));
  if (n == 0) return true;
  DevBuf<double> ad((size_t)n * n), dd(n), vd((size_t)n * n);
  DevBuf<int> ok(1);
  KNB_CUDA(cudaMemcpyAsync(ad.get(), a, (size_t)n * n * 8, cudaMemcpyHostToDevice, s));
  small_eigen<<<1, 32, 0, s>>>(ad.get(), n, dd.get(), vd.get(), ok.get());
  KNB_LAUNCH("small_eigen");
  int good = 0;
  KNB_CUDA(cudaMemcpyAsync(&good, ok.get(), 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaMemcpyAsync(d, dd.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaMemcpyAsync(V, vd.get(), (size_t)n * n * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  return good != 0;
}

}  // namespace knb
