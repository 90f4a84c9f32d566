// Katz and Bonacich power centrality on the device (reference:
// crates/engine/src/metrics/spectral.rs:300-672).
//
// Both solve the attenuated series x = b + t A x by fixed-point iteration
// (solve_series, spectral.rs:409-445) once an attenuation check
// (check_attenuation, spectral.rs:447-527) has shown that t times the
// spectral radius of A is below 1 and returned a bound q on it, from which
// the stopping rule takes the factor q / (1 - q).
//
// The check follows the reference component by component: the components
// are the strong components of the operator's positive entries (directed
// graphs) or the weak components of the graph (undirected); a single node
// is bounded by its diagonal; a larger component by Collatz ratios of power
// iteration on its own submatrix plus the identity, until the largest ratio
// falls below 1 / t (decided) or the smallest reaches it (the series
// diverges). Here all larger components iterate at once: one sweep over
// the operator with every entry that leaves its component masked to zero
// gives each component's product, and segmented reductions over the nodes
// of each component give its smallest ratio, largest ratio and largest
// entry of y + x; a decided component stops changing.
//
// The series sweep is the merge-path warp-tile kernel with an epilogue
// computing y = b + t s (no fused multiply-add, as the reference), the
// largest |y - x| and the largest |y| (fixed-order maxima), and the
// reference's stopping test in its last CTA. Bonacich power centrality
// falls back, as the reference does, to dense elimination with partial
// pivoting (I - t A) y = A 1 when the check fails, for at most 5,000 nodes;
// the elimination runs on the device in the reference's operation order.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "eigen.cuh"
#include "katz.cuh"

namespace knb {

namespace {

constexpr int KT = 256;
constexpr int K_IPT = 4;   // FP64 sweeps: 4 merge-path items per lane
constexpr int K_WPB = 16;  // 16 warps per CTA
constexpr uint32_t CHUNK = 4096;

std::string fmt(double v) {
  char b[64];
  snprintf(b, sizeof b, "%.17g", v);
  return b;
}

Error too_large(const char* name, double t, double lambda) {
  return Error(std::string(name) + " = " + fmt(t) +
               " is not below 1 / lambda_max: the largest eigenvalue of the adjacency matrix is "
               "at least " + fmt(lambda) + ", so 1 / lambda_max is at most " + fmt(1.0 / lambda));
}

// The operator a measure follows (spectral.rs:174-208): rows into a node
// (mode 2), out of it (1), or both ways (3, and undirected graphs).
struct Rows {
  int which;   // GraphHandleImpl::op rows: 0 out / undirected, 1 in, 2 directions ignored
  double lf;   // diagonal factor of a self-loop (eigenvector.rs:163-169)
  bool all;    // both directions
};
Rows rows_for(const GraphHandleImpl& g, int mode, int loops) {
  const int m = g.directed ? mode : 3;
  const bool hdir = g.directed && m != 3;
  Rows r;
  r.which = !g.directed ? 0 : (m == 3 ? 2 : (m == 2 ? 1 : 0));
  r.lf = loops == 2 ? 0.0 : (!hdir && loops == 0 ? 2.0 : 1.0);
  r.all = m == 3;
  return r;
}

// ----------------------------------------------------------------- kernels
__device__ __forceinline__ unsigned long long dbits(double v) {
  return (unsigned long long)__double_as_longlong(v);
}

__global__ void fill_d(double* x, uint32_t n, double v) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = v;
}

// Entries inside a component of two or more nodes keep their value; the
// rest become 0 (the product of a component's own submatrix).
// One warp per row.
__global__ void mask_values(OpView<double> op, const uint32_t* __restrict__ comp,
                            const uint8_t* __restrict__ big, double* __restrict__ mv) {
  const uint32_t lane = threadIdx.x & 31, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < op.n; v += nw) {
    const uint32_t c = comp[v];
    const bool keep = big[c] != 0;
    for (uint32_t k = op.off[v] + lane; k < op.off[v + 1]; k += 32)
      mv[k] = (keep && comp[op.cols[k]] == c) ? (op.vals ? op.vals[k] : 1.0) : 0.0;
  }
}

// Collatz step, per row of a component still being iterated: the ratio
// (A x)_i / x_i and y_i = (A x)_i + x_i.
struct CollatzEpi {
  static constexpr int NACC = 0;
  const uint32_t* comp;
  const uint8_t* active;
  const double* x;
  double* ratio;
  double* ynext;
  __device__ __forceinline__ void prepare(const IterState*) {}
  static __device__ __forceinline__ void init(double*) {}
  static __device__ __forceinline__ double identity(int) { return 0.0; }
  static __device__ __forceinline__ double combine(int, double a, double) { return a; }
  static __device__ __forceinline__ double warp_combine(int, double v) { return v; }
  __device__ __forceinline__ void row(uint32_t g, double s, double*) const {
    if (!active[comp[g]]) return;
    const double xg = x[g];
    ratio[g] = s / xg;
    ynext[g] = s + xg;
  }
  __device__ void finish(IterState*, const double*) const {}
};

// Per chunk of a component's nodes: smallest ratio, largest ratio, largest
// y + x (order-free extrema, so the result does not depend on the split).
__global__ void chunk_extrema(const uint32_t* __restrict__ members,
                              const uint32_t* __restrict__ chunk_comp,
                              const uint32_t* __restrict__ chunk_lo,
                              const uint32_t* __restrict__ chunk_hi,
                              const uint8_t* __restrict__ active, const double* __restrict__ ratio,
                              const double* __restrict__ ynext, uint32_t nchunks,
                              double* __restrict__ out) {
  __shared__ double s_lo[KT / 32], s_hi[KT / 32], s_top[KT / 32];
  for (uint32_t q = blockIdx.x; q < nchunks; q += gridDim.x) {
    if (!active[chunk_comp[q]]) continue;
    double lo = INFINITY, hi = 0.0, top = 0.0;
    for (uint32_t j = chunk_lo[q] + threadIdx.x; j < chunk_hi[q]; j += blockDim.x) {
      const uint32_t v = members[j];
      lo = fmin(lo, ratio[v]);
      hi = fmax(hi, ratio[v]);
      top = fmax(top, ynext[v]);
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
      top = fmax(top, __shfl_xor_sync(0xffffffffu, top, o));
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) {
      s_lo[w] = lo;
      s_hi[w] = hi;
      s_top[w] = top;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int k = 1; k < KT / 32; ++k) {
        lo = fmin(lo, s_lo[k]);
        hi = fmax(hi, s_hi[k]);
        top = fmax(top, s_top[k]);
      }
      out[(size_t)q * 3] = fmin(lo, s_lo[0]);
      out[(size_t)q * 3 + 1] = fmax(hi, s_hi[0]);
      out[(size_t)q * 3 + 2] = fmax(top, s_top[0]);
    }
  }
}

// Per component still iterated: joins its chunks and decides. status: 0
// iterating, 1 decided (hi < limit; bound in value), 2 diverges (lo >=
// limit; lo in value).
__global__ void collatz_decide(const uint32_t* __restrict__ big_comps, uint32_t nbig,
                               const uint32_t* __restrict__ comp_chunk0,
                               const double* __restrict__ cx, double limit,
                               uint8_t* __restrict__ active, uint8_t* __restrict__ status,
                               double* __restrict__ value, double* __restrict__ top) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nbig; b += gridDim.x * blockDim.x) {
    const uint32_t c = big_comps[b];
    if (!active[c]) continue;
    double lo = INFINITY, hi = 0.0, tp = 0.0;
    for (uint32_t q = comp_chunk0[b]; q < comp_chunk0[b + 1]; ++q) {
      lo = fmin(lo, cx[(size_t)q * 3]);
      hi = fmax(hi, cx[(size_t)q * 3 + 1]);
      tp = fmax(tp, cx[(size_t)q * 3 + 2]);
    }
    if (lo >= limit) {
      status[b] = 2;
      value[b] = lo;
      active[c] = 0;
    } else if (hi < limit) {
      status[b] = 1;
      value[b] = hi;
      active[c] = 0;
    } else {
      top[c] = tp;
    }
  }
}

__global__ void collatz_next(const uint32_t* __restrict__ comp, const uint8_t* __restrict__ active,
                             const double* __restrict__ ynext, const double* __restrict__ top,
                             uint32_t n, double* __restrict__ x) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t c = comp[i];
    if (active[c]) x[i] = ynext[i] / top[c];
  }
}

// Series step y = b + t s; the largest |y - x| and |y|; the reference's
// stopping test (spectral.rs:429-441) in the last CTA.
struct SeriesEpi {
  static constexpr int NACC = 2;
  const double* b;
  const double* x_old;
  double* y_new;
  double t;
  double factor;
  __device__ __forceinline__ void prepare(const IterState*) {}
  static __device__ __forceinline__ void init(double* a) { a[0] = a[1] = 0.0; }
  static __device__ __forceinline__ double identity(int) { return 0.0; }
  static __device__ __forceinline__ double combine(int, double a, double c) { return fmax(a, c); }
  static __device__ __forceinline__ double warp_combine(int, double v) { return warp_max(v); }
  __device__ __forceinline__ void row(uint32_t g, double s, double* a) const {
    const double y = __dadd_rn(b[g], __dmul_rn(t, s));
    y_new[g] = y;
    a[0] = fmax(a[0], fabs(y - x_old[g]));
    a[1] = fmax(a[1], fabs(y));
  }
  __device__ void finish(IterState* st, const double* tot) const {
    st->change = tot[0];
    st->top = tot[1];
    st->iter += 1;
    if (tot[0] * factor <= st->tol * tot[1] || tot[1] == 0.0) st->converged = 1;
    else if (st->iter >= st->max_iter) st->stopped = 1;
  }
};

// Row sums b = A 1 in row order (SparseOp::apply on ones).
__global__ void row_sums(OpView<double> op, double* __restrict__ b) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < op.n; v += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (uint32_t k = op.off[v]; k < op.off[v + 1]; ++k) s += op.vals ? op.vals[k] : 1.0;
    b[v] = s;
  }
}

// ----------------------------------------------------------------- dense solve
// Gaussian elimination with partial pivoting on (I - t A) y = b, in the
// order of linalg.rs:433-467 (first row of largest magnitude as pivot; a
// pivot at most 1e-12 times the largest magnitude of the matrix is
// singular).
struct DenseState {
  unsigned long long absmax;  // bits of the largest |a_ij|
  uint32_t pivot;
  int32_t singular;
};

__global__ void dense_identity(double* a, uint32_t n) {
  const size_t nn = (size_t)n * n;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nn;
       q += (size_t)gridDim.x * blockDim.x)
    a[q] = (q / n == q % n) ? 1.0 : 0.0;
}

__global__ void dense_scatter(OpView<double> op, double t, double* a) {
  const size_t n = op.n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < op.n; i += gridDim.x * blockDim.x)
    for (uint32_t k = op.off[i]; k < op.off[i + 1]; ++k) {
      double& e = a[(size_t)i * n + op.cols[k]];
      e = __dsub_rn(e, __dmul_rn(t, op.vals ? op.vals[k] : 1.0));
    }
}

__global__ void dense_absmax(const double* a, size_t nn, DenseState* ds) {
  double m = 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < nn;
       q += (size_t)gridDim.x * blockDim.x)
    m = fmax(m, fabs(a[q]));
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) atomicMax(&ds->absmax, dbits(m));
}

__global__ void dense_pivot(const double* a, uint32_t n, uint32_t k, DenseState* ds) {
  __shared__ double sv[KT / 32];
  __shared__ uint32_t si[KT / 32];
  if (ds->singular) return;
  double best = -1.0;
  uint32_t bi = n;
  for (uint32_t r = k + threadIdx.x; r < n; r += blockDim.x) {
    const double v = fabs(a[(size_t)r * n + k]);
    if (v > best) {
      best = v;
      bi = r;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const double ov = __shfl_xor_sync(0xffffffffu, best, o);
    const uint32_t oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov > best || (ov == best && oi < bi)) {
      best = ov;
      bi = oi;
    }
  }
  if ((threadIdx.x & 31) == 0) {
    sv[threadIdx.x >> 5] = best;
    si[threadIdx.x >> 5] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < KT / 32; ++w)
      if (sv[w] > best || (sv[w] == best && si[w] < bi)) {
        best = sv[w];
        bi = si[w];
      }
    const double mag = fmax(__longlong_as_double((long long)ds->absmax), DBL_MIN);
    ds->pivot = bi;
    if (!(best > 1e-12 * mag)) ds->singular = 1;
  }
}

__global__ void dense_swap(double* a, double* x, uint32_t n, uint32_t k, const DenseState* ds) {
  if (ds->singular) return;
  const uint32_t p = ds->pivot;
  if (p == k) return;
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
    const double u = a[(size_t)k * n + c];
    a[(size_t)k * n + c] = a[(size_t)p * n + c];
    a[(size_t)p * n + c] = u;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const double u = x[k];
    x[k] = x[p];
    x[p] = u;
  }
}

// One CTA per row i > k: f = a_ik / a_kk; a_ij -= f a_kj (j > k); x_i -= f x_k.
__global__ void dense_eliminate(double* a, double* x, uint32_t n, uint32_t k,
                                const DenseState* ds) {
  if (ds->singular) return;
  for (uint32_t i = k + 1 + blockIdx.x; i < n; i += gridDim.x) {
    const double f = a[(size_t)i * n + k] / a[(size_t)k * n + k];
    if (f == 0.0) continue;
    for (uint32_t j = k + 1 + threadIdx.x; j < n; j += blockDim.x)
      a[(size_t)i * n + j] = __dsub_rn(a[(size_t)i * n + j], __dmul_rn(f, a[(size_t)k * n + j]));
    __syncthreads();
    if (threadIdx.x == 0) {
      a[(size_t)i * n + k] = 0.0;
      x[i] = __dsub_rn(x[i], __dmul_rn(f, x[k]));
    }
    __syncthreads();
  }
}

// Back substitution in one CTA: x_k = (x_k - sum_{j > k} a_kj x_j) / a_kk,
// the sum in a fixed order.
__global__ void dense_back(const double* a, double* x, uint32_t n, const DenseState* ds) {
  __shared__ double part[1024 / 32];
  if (ds->singular) return;
  for (uint32_t kk = n; kk-- > 0;) {
    double s = 0.0;
    for (uint32_t j = kk + 1 + threadIdx.x; j < n; j += blockDim.x)
      s += a[(size_t)kk * n + j] * x[j];
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (uint32_t w = 0; w < blockDim.x / 32; ++w) t += part[w];
      x[kk] = (x[kk] - t) / a[(size_t)kk * n + kk];
    }
    __syncthreads();
  }
}

// ----------------------------------------------------------------- host parts
template <class Epi>
void sweep(const OpView<double>& v, const Partition& P, const double* x, const Epi& e,
           double* carry, double* head, double* part1, double* part2, IterState* st,
           cudaStream_t s) {
  constexpr size_t smem = warp_smem_bytes<double, K_IPT, K_WPB>();
  const unsigned grid = (P.ntiles + K_WPB - 1) / K_WPB;
  fit_warp_carveout<double, double, Epi, K_IPT, K_WPB>();
  warp_spmv<double, double, Epi, K_IPT, K_WPB><<<grid, K_WPB * 32, smem, s>>>(
      v, x, e, P.coords.get(), P.ntiles, carry, head, part1, st, 0xFFFFFFFFu);
  KNB_LAUNCH("series sweep");
  split_rows<double, Epi><<<SPLIT_CTAS, SPMV_THREADS, 0, s>>>(
      P.split.get(), P.nsplit, P.nshort, carry, head, e, part1, P.ntiles, part2, st);
  KNB_LAUNCH("series split rows");
}

struct Scratch {
  DevBuf<double> carry, head, part1, part2;
  DevBuf<IterState> st;
  explicit Scratch(const Partition& P)
      : carry(P.ntiles + 1), head(P.ntiles + 1), part1((size_t)P.ntiles * 2 + 2),
        part2((size_t)SPLIT_CTAS * 2 + 2), st(1) {}
};

// A node's diagonal entry: the sum of its self-loop values (weight, or 1,
// times the loop factor) in input order. Rows of the out-CSR are sorted by
// target with ties in input order, so a thread finds its loops by binary
// search and adds them in that order.
__global__ void loop_diag(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                          const double* __restrict__ w, uint32_t n, double lf,
                          double* __restrict__ diag) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t lo = off[i], hi = off[i + 1];
    const uint32_t end = hi;
    while (lo < hi) {
      const uint32_t mid = lo + ((hi - lo) >> 1);
      if (tgt[mid] < i) lo = mid + 1; else hi = mid;
    }
    double d = 0.0;
    for (uint32_t k = lo; k < end && tgt[k] == i; ++k)
      d = __dadd_rn(d, __dmul_rn(w ? w[k] : 1.0, lf));
    diag[i] = d;
  }
}

// What the attenuation check on one operator can reuse whatever t is: the
// components, the diagonal of every single-node component (in label order),
// the larger components' member lists and chunks, and the operator with the
// entries that leave their component masked to 0. Held for the length of a
// check, so concurrent calls on one operator take turns.
struct SeriesPlan : Workspace {
  std::mutex mu;
  bool ready = false;
  size_t k = 0;
  std::vector<double> single_diag;
  uint32_t nbig = 0, nch = 0;
  DevBuf<uint32_t> d_comp, d_members, d_big, d_cc0, d_chc, d_chl, d_chh;
  DevBuf<uint8_t> d_big_flags;
  DevBuf<double> mv;
};

static void series_prepare(SeriesPlan& plan, GraphHandleImpl& g, const Operator& op,
                           const Rows& rw, bool weighted, cudaStream_t s) {
  const uint32_t n = g.n;
  Comps comp;
  if (g.directed) {
    // strong components of the positive entries (spectral.rs:539-553); a
    // loop's factor leaves the pattern of the other entries as it is
    comp = strong_components(g, weighted ? g.w.get() : nullptr, rw.all, nullptr, s);
  } else {
    comp = weak_components(g, s);
  }
  const size_t k = comp.count();
  plan.k = k;
  // single nodes: the diagonal (the sum of a node's self-loop entries)
  std::vector<double> diag(n, 0.0);
  if (n) {
    DevBuf<double> dd(n);
    loop_diag<<<grid_for(n, KT), KT, 0, s>>>(g.out.off.get(), g.out.tgt.get(),
                                              weighted ? g.out.w.get() : nullptr, n, rw.lf,
                                              dd.get());
    KNB_LAUNCH("loop_diag");
    KNB_CUDA(cudaMemcpyAsync(diag.data(), dd.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
  }
  std::vector<uint32_t> first(k, 0xFFFFFFFFu);
  for (uint32_t v = 0; v < n; ++v)
    if (first[comp.membership[v]] == 0xFFFFFFFFu) first[comp.membership[v]] = v;
  plan.single_diag.clear();
  for (size_t c = 0; c < k; ++c)
    if (comp.sizes[c] == 1) plan.single_diag.push_back(diag[first[c]]);
  // larger components: nodes grouped by component, chunks of CHUNK nodes
  std::vector<uint32_t> big_comps, comp_chunk0, members, chunk_comp, chunk_lo, chunk_hi;
  std::vector<uint32_t> start(k + 1, 0);
  for (size_t c = 0; c < k; ++c) start[c + 1] = start[c] + (comp.sizes[c] > 1 ? comp.sizes[c] : 0);
  members.resize(start[k]);
  {
    std::vector<uint32_t> cur(start.begin(), start.end() - 1);
    for (uint32_t v = 0; v < n; ++v) {
      const uint32_t c = comp.membership[v];
      if (comp.sizes[c] > 1) members[cur[c]++] = v;
    }
  }
  std::vector<uint8_t> big(k, 0);
  for (size_t c = 0; c < k; ++c)
    if (comp.sizes[c] > 1) {
      big[c] = 1;
      big_comps.push_back((uint32_t)c);
      comp_chunk0.push_back((uint32_t)chunk_comp.size());
      for (uint32_t a = start[c]; a < start[c + 1]; a += CHUNK) {
        chunk_comp.push_back((uint32_t)c);
        chunk_lo.push_back(a);
        chunk_hi.push_back(std::min(start[c + 1], a + CHUNK));
      }
    }
  comp_chunk0.push_back((uint32_t)chunk_comp.size());
  plan.nbig = (uint32_t)big_comps.size();
  plan.nch = (uint32_t)chunk_comp.size();
  if (plan.nbig) {
    auto up32 = [&](DevBuf<uint32_t>& d, const std::vector<uint32_t>& h) {
      d.alloc(std::max<size_t>(h.size(), 1));
      if (!h.empty())
        KNB_CUDA(cudaMemcpyAsync(d.get(), h.data(), h.size() * 4, cudaMemcpyHostToDevice, s));
    };
    up32(plan.d_comp, comp.membership);
    up32(plan.d_members, members);
    up32(plan.d_big, big_comps);
    up32(plan.d_cc0, comp_chunk0);
    up32(plan.d_chc, chunk_comp);
    up32(plan.d_chl, chunk_lo);
    up32(plan.d_chh, chunk_hi);
    plan.d_big_flags.alloc(std::max<size_t>(k, 1));
    KNB_CUDA(cudaMemcpyAsync(plan.d_big_flags.get(), big.data(), k, cudaMemcpyHostToDevice, s));
    plan.mv.alloc(std::max<uint64_t>(op.nnz, 1));
    const OpView<double> v0 = op.view64();
    mask_values<<<grid_for((uint64_t)n * 32, KT), KT, 0, s>>>(v0, plan.d_comp.get(),
                                                            plan.d_big_flags.get(), plan.mv.get());
    KNB_LAUNCH("collatz set-up");
    KNB_CUDA(cudaStreamSynchronize(s));
  }
  plan.ready = true;
}

// check_attenuation (spectral.rs:447-527): returns the radius bound or
// throws. `collatz` receives the number of power-iteration steps.
double attenuation_bound(GraphHandleImpl& g, const Operator& op, const Rows& rw, bool weighted,
                         double t, const char* name, int64_t max_iter, int64_t* collatz,
                         cudaStream_t s) {
  const uint32_t n = g.n;
  const double limit = 1.0 / t;
  *collatz = 0;
  Operator& mop = const_cast<Operator&>(op);
  SeriesPlan* planp = nullptr;
  {
    std::lock_guard<std::mutex> lock(mop.mu);
    if (!mop.series_ws) mop.series_ws = std::make_unique<SeriesPlan>();
    planp = static_cast<SeriesPlan*>(mop.series_ws.get());
  }
  SeriesPlan& plan = *planp;
  std::lock_guard<std::mutex> plan_lock(plan.mu);
  if (!plan.ready) series_prepare(plan, g, op, rw, weighted, s);
  double radius = 0.0;
  for (double d : plan.single_diag) {
    if (d >= limit) throw too_large(name, t, d);
    radius = std::max(radius, d);
  }
  if (plan.nbig == 0) return radius;
  const size_t k = plan.k;
  const uint32_t nbig = plan.nbig, nch = plan.nch;
  DevBuf<uint8_t> d_active(k), d_status(nbig);
  KNB_CUDA(cudaMemcpyAsync(d_active.get(), plan.d_big_flags.get(), k, cudaMemcpyDeviceToDevice, s));
  KNB_CUDA(cudaMemsetAsync(d_status.get(), 0, nbig, s));
  DevBuf<double> x(n), ratio(n), ynext(n), cx((size_t)nch * 3), value_b(nbig), top(k);
  const OpView<double> v0 = op.view64();
  fill_d<<<grid_for(n, KT), KT, 0, s>>>(x.get(), n, 1.0);
  KNB_LAUNCH("collatz start");
  const OpView<double> vm{v0.n, v0.nnz, v0.off, v0.cols, plan.mv.get()};
  const Partition& P = mop.partition(32 * K_IPT, s);
  Scratch sc(P);
  CollatzEpi e{plan.d_comp.get(), d_active.get(), x.get(), ratio.get(), ynext.get()};
  std::vector<uint8_t> status(nbig, 0);
  std::vector<double> vals(nbig, 0.0);
  bool done = false;
  for (int64_t it = 0; it < max_iter && !done; ++it) {
    sweep(vm, P, x.get(), e, sc.carry.get(), sc.head.get(), sc.part1.get(), sc.part2.get(),
          nullptr, s);
    chunk_extrema<<<std::min<uint32_t>(nch, 148 * 8), KT, 0, s>>>(
        plan.d_members.get(), plan.d_chc.get(), plan.d_chl.get(), plan.d_chh.get(),
        d_active.get(), ratio.get(), ynext.get(), nch, cx.get());
    collatz_decide<<<grid_for(nbig, KT), KT, 0, s>>>(plan.d_big.get(), nbig, plan.d_cc0.get(),
                                                     cx.get(), limit, d_active.get(),
                                                     d_status.get(), value_b.get(), top.get());
    collatz_next<<<grid_for(n, KT), KT, 0, s>>>(plan.d_comp.get(), d_active.get(), ynext.get(),
                                                top.get(), n, x.get());
    KNB_LAUNCH("collatz step");
    *collatz = it + 1;
    KNB_CUDA(cudaMemcpyAsync(status.data(), d_status.get(), nbig, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    done = true;
    for (uint32_t b = 0; b < nbig; ++b)
      if (status[b] != 1) done = false;
    for (uint32_t b = 0; b < nbig; ++b)
      if (status[b] == 2) {  // the first component (by label) whose series diverges
        KNB_CUDA(cudaMemcpy(vals.data(), value_b.get(), (size_t)nbig * 8, cudaMemcpyDeviceToHost));
        throw too_large(name, t, vals[b]);
      }
  }
  if (!done)
    throw Error(std::string(name) + " = " + fmt(t) +
                " is too close to 1 / lambda_max to decide whether the series converges; "
                "choose a smaller value");
  KNB_CUDA(cudaMemcpy(vals.data(), value_b.get(), (size_t)nbig * 8, cudaMemcpyDeviceToHost));
  for (uint32_t b = 0; b < nbig; ++b) radius = std::max(radius, vals[b]);
  return radius;
}

// solve_series (spectral.rs:409-445) from x = b (device); returns the
// device buffer holding the result (x or y) and the sweep count.
const double* series(const Operator& op, const double* d_b, double t, double q, double tol,
                     int64_t max_iter, const char* what, DevBuf<double> (&xb)[2], int64_t* iters,
                     cudaStream_t s) {
  const uint32_t n = op.n;
  KNB_CUDA(cudaMemcpyAsync(xb[0].get(), d_b, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
  *iters = 0;
  if (t == 0.0) return xb[0].get();
  const Partition& P = const_cast<Operator&>(op).partition(32 * K_IPT, s);
  Scratch sc(P);
  IterState is{};
  is.tol = tol;
  is.max_iter = (int32_t)std::min<int64_t>(max_iter, INT32_MAX);
  KNB_CUDA(cudaMemcpyAsync(sc.st.get(), &is, sizeof(is), cudaMemcpyHostToDevice, s));
  const OpView<double> v = op.view64();
  SeriesEpi e;
  e.b = d_b;
  e.t = t;
  e.factor = std::max(q / (1.0 - q), 1.0);
  IterState hs{};
  for (;;) {
    for (int k = 0; k < 8; ++k) {
      e.x_old = xb[k & 1].get();
      e.y_new = xb[1 - (k & 1)].get();
      sweep(v, P, xb[k & 1].get(), e, sc.carry.get(), sc.head.get(), sc.part1.get(),
            sc.part2.get(), sc.st.get(), s);
    }
    KNB_CUDA(cudaMemcpyAsync(&hs, sc.st.get(), sizeof(hs), cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    if (hs.converged || hs.stopped) break;
  }
  *iters = hs.iter;
  if (!hs.converged)
    throw Error(std::string(what) + " did not converge to tolerance " + fmt(tol) + " within " +
                std::to_string(max_iter) + " iterations");
  return xb[hs.iter & 1].get();
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

void katz(GraphHandleImpl& g, double alpha, const std::vector<double>& beta, bool normalized,
          const SeriesParams& p, double* out, SeriesResult* r, cudaStream_t s) {
  const auto t0 = std::chrono::steady_clock::now();
  const uint32_t n = g.n;
  if (n == 0) return;
  const Rows rw = rows_for(g, p.mode, p.loops);
  Operator& op = g.op(rw.which, p.weighted, rw.lf, s);
  const double q = alpha > 0.0 ? alpha * attenuation_bound(g, op, rw, p.weighted, alpha, "alpha",
                                                           p.max_iter, &r->collatz, s)
                               : 0.0;
  r->radius = alpha > 0.0 ? q / alpha : 0.0;
  DevBuf<double> b(n), xb[2] = {DevBuf<double>(n), DevBuf<double>(n)};
  KNB_CUDA(cudaMemcpyAsync(b.get(), beta.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
  const double* x = series(op, b.get(), alpha, q, p.tol, p.max_iter, "Katz centrality", xb,
                           &r->iterations, s);
  KNB_CUDA(cudaMemcpyAsync(out, x, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  if (normalized) {
    double ss = 0.0;
    for (uint32_t i = 0; i < n; ++i) ss += out[i] * out[i];
    const double norm = std::sqrt(ss);
    if (norm > 0.0)
      for (uint32_t i = 0; i < n; ++i) out[i] /= norm;
  }
  r->seconds = seconds_since(t0);
}

void bonacich_power(GraphHandleImpl& g, double exponent, bool rescale, const SeriesParams& p,
                    double* out, SeriesResult* r, cudaStream_t s) {
  const auto t0 = std::chrono::steady_clock::now();
  const uint32_t n = g.n;
  if (n == 0) return;
  const Rows rw = rows_for(g, p.mode, p.loops);
  Operator& op = g.op(rw.which, p.weighted, rw.lf, s);
  const OpView<double> v = op.view64();
  DevBuf<double> b(n), xb[2] = {DevBuf<double>(n), DevBuf<double>(n)};
  row_sums<<<grid_for(n, KT), KT, 0, s>>>(v, b.get());
  KNB_LAUNCH("row_sums");
  const double beta = exponent;
  bool use_series = true;
  double q = 0.0;
  if (beta != 0.0) {
    try {
      q = attenuation_bound(g, op, rw, p.weighted, std::fabs(beta), "|exponent|", p.max_iter,
                            &r->collatz, s) * std::fabs(beta);
    } catch (const Error&) {
      use_series = false;
    }
  }
  if (use_series) {
    const double* y = series(op, b.get(), beta, q, p.tol, p.max_iter, "power centrality", xb,
                             &r->iterations, s);
    KNB_CUDA(cudaMemcpyAsync(out, y, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  } else {
    if (n > 5000)
      throw Error("|exponent| x lambda_max >= 1, so power centrality needs a dense linear solve, "
                  "which is limited to 5000 nodes; use a smaller |exponent|");
    const size_t nn = (size_t)n * n;
    DevBuf<double> a(nn);
    DevBuf<DenseState> ds(1);
    KNB_CUDA(cudaMemsetAsync(ds.get(), 0, sizeof(DenseState), s));
    dense_identity<<<grid_for(nn, KT), KT, 0, s>>>(a.get(), n);
    dense_scatter<<<grid_for(n, KT), KT, 0, s>>>(v, beta, a.get());
    dense_absmax<<<grid_for(nn, KT), KT, 0, s>>>(a.get(), nn, ds.get());
    KNB_LAUNCH("dense set-up");
    double* x = b.get();  // the right-hand side, solved in place
    for (uint32_t k = 0; k < n; ++k) {
      dense_pivot<<<1, KT, 0, s>>>(a.get(), n, k, ds.get());
      dense_swap<<<grid_for(n, KT, 64), KT, 0, s>>>(a.get(), x, n, k, ds.get());
      if (k + 1 < n)
        dense_eliminate<<<std::min<uint32_t>(n - k - 1, 148 * 8), KT, 0, s>>>(a.get(), x, n, k,
                                                                               ds.get());
    }
    KNB_LAUNCH("dense elimination");
    dense_back<<<1, 1024, 0, s>>>(a.get(), x, n, ds.get());
    KNB_LAUNCH("dense back substitution");
    DenseState h{};
    KNB_CUDA(cudaMemcpyAsync(&h, ds.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaMemcpyAsync(out, x, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    if (h.singular)
      throw Error("I - exponent x A is singular (exponent is the reciprocal of an eigenvalue), so "
                  "power centrality is undefined; choose another exponent");
    r->dense = true;
  }
  KNB_CUDA(cudaStreamSynchronize(s));
  double sq = 0.0;
  for (uint32_t i = 0; i < n; ++i) sq += out[i] * out[i];
  const double alpha = std::sqrt((double)n / sq);
  if (rescale) {
    double total = 0.0;
    for (uint32_t i = 0; i < n; ++i) total += out[i];
    for (uint32_t i = 0; i < n; ++i) out[i] /= total;
  } else {
    for (uint32_t i = 0; i < n; ++i) out[i] *= alpha;
  }
  r->seconds = seconds_since(t0);
}

}  // namespace knb
