// Differentiable PageRank: PageRank of caller-supplied edge weights, and the
// gradient of a loss L(x) with respect to those weights.
//
// At the fixed point, x = d (M x + jump 1_D^T x) + (1 - d) p with 1^T x = 1,
// where M_ij = sum of f_e w_e over arcs e = (j -> i), divided by the
// out-strength s_j, f_e the self-loop factor, and D the dangling nodes
// (s_j = 0). With A = I - d M - d jump 1_D^T (invertible for d < 1: the
// matrix d (M + jump 1_D^T) is d times a column-stochastic matrix) and
// g = dL/dx, the adjoint lambda solves A^T lambda = g, i.e.
//     lambda = g + d M^T lambda + d 1_D (jump^T lambda),
// a fixed-point iteration that contracts by d in the max norm. It pulls along
// out-arcs: (M^T lambda)_j = sum over arcs (j -> i) of f_e w_e lambda_i / s_j,
// so it runs on the merge-path sweep over the out-adjacency. Then, since
// dM_kj/dw_e = f_e (delta_ki - M_kj) / s_j for e = (j -> i),
//     dL/dw_e = d f_e (x_j / s_j) (lambda_i - (M^T lambda)_j),
// the second term being the derivative of the row (out-strength)
// normalisation. An undirected edge adds the terms of its two arcs. Dangling
// nodes stay dangling for positive weights, so D does not move.
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "adjoint.cuh"
#include "pagerank.cuh"

namespace knb {

struct AdjointEpi {
  static constexpr int NACC = 2;
  const double* g;
  const double* lam_old;
  double* lam_new;
  const double* inv_out;
  const double* jump;  // null: uniform
  double d, pu;
  double jdot = 0;

  __device__ __forceinline__ void prepare(const IterState* st) { jdot = st ? st->dterm : 0.0; }
  static __device__ __forceinline__ void init(double* a) { a[0] = a[1] = 0.0; }
  static __device__ __forceinline__ double identity(int) { return 0.0; }
  static __device__ __forceinline__ double combine(int, double a, double b) { return a + b; }
  static __device__ __forceinline__ double warp_combine(int, double v) { return warp_sum(v); }
  __device__ __forceinline__ void row(uint32_t j, double r, double* a) const {
    const double io = inv_out[j];
    const double v = g[j] + d * (io > 0.0 ? r * io : jdot);
    lam_new[j] = v;
    a[0] += fabs(v - lam_old[j]);
    a[1] += (jump ? jump[j] : pu) * v;
  }
  __device__ void finish(IterState* st, const double* tot) const {
    st->change = tot[0];
    st->dterm = tot[1];
    st->iter += 1;
    if (tot[0] <= st->tol) st->converged = 1;
    else if (st->iter >= st->max_iter) st->stopped = 1;
  }
};

// Row sums r_j = sum of f_e w_e lambda_i (final lambda), stored.
struct RowSumEpi {
  static constexpr int NACC = 0;
  double* r;
  __device__ __forceinline__ void prepare(const IterState*) {}
  static __device__ __forceinline__ void init(double*) {}
  static __device__ __forceinline__ double identity(int) { return 0.0; }
  static __device__ __forceinline__ double combine(int, double a, double b) { return a + b; }
  static __device__ __forceinline__ double warp_combine(int, double v) { return v; }
  __device__ __forceinline__ void row(uint32_t j, double s, double*) const { r[j] = s; }
  __device__ void finish(IterState*, const double*) const {}
};

__global__ void adj_init(const double* __restrict__ g, const double* __restrict__ jump, uint32_t n,
                         double* __restrict__ lam, double* __restrict__ part, IterState* st) {
  __shared__ double sh[8];
  double a = 0;
  const double pu = 1.0 / n;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    lam[i] = g[i];
    a += (jump ? jump[i] : pu) * g[i];
  }
  a = block_sum(a, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = a;
  __threadfence();
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(&st->ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  double t = 0;
  for (uint32_t q = threadIdx.x; q < gridDim.x; q += blockDim.x) t += __ldcg(part + q);
  t = block_sum(t, sh);
  if (threadIdx.x == 0) {
    st->dterm = t;
    st->ticket = 0;
  }
}

// dL/dw_e over the arcs of the out-adjacency (row j = source).
__global__ void adj_grad(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                         const uint32_t* __restrict__ edge, uint32_t n, double lf, double d,
                         const double* __restrict__ x, const double* __restrict__ inv_out,
                         const double* __restrict__ lam, const double* __restrict__ r,
                         int two_arcs, double* __restrict__ grad) {
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const double io = inv_out[j];
    if (!(io > 0.0)) continue;  // no out-arcs of positive weight: nothing depends on them
    const double xs = x[j] * io, mt = r[j] * io;
    for (uint32_t k = off[j]; k < off[j + 1]; ++k) {
      const uint32_t i = tgt[k];
      const double f = i == j ? lf : 1.0;
      const double gv = d * f * xs * (lam[i] - mt);
      if (two_arcs) atomicAdd(grad + edge[k], gv);  // at most two terms: order-free
      else grad[edge[k]] = gv;
    }
  }
}

static void normalized_jump(const double* d_pers, uint32_t n, DevBuf<double>& out,
                            cudaStream_t s) {
  std::vector<double> h(n);
  KNB_CUDA(cudaMemcpyAsync(h.data(), d_pers, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  double t = 0;
  for (double v : h) {
    if (!std::isfinite(v) || v < 0.0)
      throw Error("the personalization vector must hold finite, nonnegative values");
    t += v;
  }
  if (!(t > 0.0)) throw Error("the personalization vector must have a positive sum");
  for (double& v : h) v /= t;
  out.alloc(n);
  KNB_CUDA(cudaMemcpyAsync(out.get(), h.data(), (size_t)n * 8, cudaMemcpyHostToDevice, s));
}

void pagerank_weights(GraphHandleImpl& g, const double* d_w, const PagerankParams& prm,
                      double* d_out, PagerankInfo* info, cudaStream_t s) {
  if (g.n == 0) return;
  const int which = pagerank_rows(g, prm.directed);
  const double lf = pagerank_loop_factor(which, prm.loops);
  GraphHandleImpl::WeightSlot& slot = g.weight_slot(which, lf, s);
  std::lock_guard<std::mutex> lock(slot.mu);
  g.fill_weights(*slot.op, d_w, lf, s);
  PagerankParams p = prm;
  p.weighted = true;
  p.relabel = false;  // values change every call: no renumbered copy
  pagerank_op(*slot.op, p, d_out, true, info, s);
}

void pagerank_grad(GraphHandleImpl& g, const double* d_w, const double* d_x, const double* d_gx,
                   const AdjointParams& prm, double* d_gw, double* d_lambda, AdjointInfo* info,
                   cudaStream_t s) {
  const uint32_t n = g.n;
  KNB_CUDA(cudaMemsetAsync(d_gw, 0, std::max<uint64_t>(g.m, 1) * 8, s));
  if (n == 0) return;
  const int which = pagerank_rows(g, prm.directed);
  const double lf = pagerank_loop_factor(which, prm.loops);
  // fwd: its column sums are the out-strengths; tr: pull along out-arcs
  const int twhich = which == 1 ? 0 : which;
  GraphHandleImpl::WeightSlot& fslot = g.weight_slot(which, lf, s);
  GraphHandleImpl::WeightSlot& tslot = g.weight_slot(twhich, lf, s);
  std::unique_lock<std::mutex> flock(fslot.mu, std::defer_lock), tlock(tslot.mu, std::defer_lock);
  if (&fslot == &tslot) flock.lock();
  else std::lock(flock, tlock);
  Operator* fwd = fslot.op.get();
  Operator* tr = tslot.op.get();
  g.fill_weights(*fwd, d_w, lf, s);
  if (tr != fwd) g.fill_weights(*tr, d_w, lf, s);
  const Partition& P = tr->partition(128, s);
  DevBuf<double> jump;
  if (prm.personalization && prm.dangling == 0) normalized_jump(prm.personalization, n, jump, s);

  // ||g||_1 scales the stopping rule
  std::vector<double> hg(n);
  KNB_CUDA(cudaMemcpyAsync(hg.data(), d_gx, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  double gnorm = 0;
  for (double v : hg) gnorm += std::fabs(v);

  DevBuf<double> lam[2] = {DevBuf<double>(n), DevBuf<double>(n)}, r(n), carry(P.ntiles + 1),
                head(P.ntiles + 1), part1((size_t)P.ntiles * 2 + 2),
                part2((size_t)SPLIT_CTAS * 2 + 2), part3(1184 + 2);
  DevBuf<IterState> st(1);
  IterState is{};
  is.tol = prm.tol * std::max(1.0, gnorm);
  is.max_iter = (int32_t)std::min<int64_t>(prm.max_iter, INT32_MAX);
  KNB_CUDA(cudaMemcpyAsync(st.get(), &is, sizeof(is), cudaMemcpyHostToDevice, s));
  cudaEvent_t t0, t1;
  KNB_CUDA(cudaEventCreate(&t0));
  KNB_CUDA(cudaEventCreate(&t1));
  KNB_CUDA(cudaEventRecord(t0, s));
  const unsigned gv = grid_for(n, 256, 1184);
  adj_init<<<gv, 256, 0, s>>>(d_gx, jump.get(), n, lam[0].get(), part3.get(), st.get());
  KNB_LAUNCH("adj_init");
  int launches = 1;
  constexpr int IPT = 4, WPB = 4;
  constexpr size_t smem = warp_smem_bytes<double, IPT, WPB>();
  const unsigned grid = (P.ntiles + WPB - 1) / WPB;
  const OpView<double> v = tr->view64();
  IterState h{};
  int k = 0;
  fit_warp_carveout<double, double, AdjointEpi, IPT, WPB>();
  fit_warp_carveout<double, double, RowSumEpi, IPT, WPB>();
  for (;;) {
    for (int b = 0; b < 8; ++b, ++k) {
      AdjointEpi e;
      e.g = d_gx;
      e.lam_old = lam[k & 1].get();
      e.lam_new = lam[1 - (k & 1)].get();
      e.inv_out = fwd->inv_out64.get();
      e.jump = jump.get();
      e.d = prm.damping;
      e.pu = 1.0 / n;
      warp_spmv<double, double, AdjointEpi, IPT, WPB><<<grid, WPB * 32, smem, s>>>(
          v, lam[k & 1].get(), e, P.coords.get(), P.ntiles, carry.get(), head.get(), part1.get(),
          st.get(), 0xFFFFFFFFu);
      split_rows<double, AdjointEpi><<<SPLIT_CTAS, SPMV_THREADS, 0, s>>>(
          P.split.get(), P.nsplit, P.nshort, carry.get(), head.get(), e, part1.get(), P.ntiles,
          part2.get(), st.get());
      launches += 2;
    }
    KNB_LAUNCH("adjoint sweep");
    KNB_CUDA(cudaMemcpyAsync(&h, st.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    if (h.converged || h.stopped) break;
  }
  if (!h.converged)
    throw Error("the PageRank adjoint did not converge within " + std::to_string(prm.max_iter) +
                " iterations");
  const double* lam_final = lam[h.iter & 1].get();
  // (M^T lambda)_j numerators with the final lambda, then the edge gradients
  {
    RowSumEpi e{r.get()};
    warp_spmv<double, double, RowSumEpi, IPT, WPB><<<grid, WPB * 32, smem, s>>>(
        v, lam_final, e, P.coords.get(), P.ntiles, carry.get(), head.get(), part1.get(), nullptr,
        0xFFFFFFFFu);
    split_rows<double, RowSumEpi><<<SPLIT_CTAS, SPMV_THREADS, 0, s>>>(
        P.split.get(), P.nsplit, P.nshort, carry.get(), head.get(), e, part1.get(), P.ntiles,
        part2.get(), nullptr);
    const DevCsr* rows = tr->rows;
    adj_grad<<<grid_for(n, 128), 128, 0, s>>>(rows->off.get(), rows->tgt.get(), rows->edge.get(),
                                              n, lf, prm.damping, d_x, fwd->inv_out64.get(),
                                              lam_final, r.get(), which != 1 ? 1 : 0,
                                              d_gw);
    launches += 3;
    KNB_LAUNCH("adjoint gradient");
  }
  if (d_lambda)
    KNB_CUDA(cudaMemcpyAsync(d_lambda, lam_final, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
  KNB_CUDA(cudaEventRecord(t1, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  KNB_CUDA(cudaEventElapsedTime(&ms, t0, t1));
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  if (info) {
    info->iterations = h.iter;
    info->change = h.change;
    info->seconds = ms * 1e-3;
    info->kernel_launches = launches;
  }
}

}  // namespace knb
