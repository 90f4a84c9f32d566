// PageRank power iteration on the device (reference: the loop of
// crates/engine/src/metrics/spectral.rs:211-281).
//
// One sweep is two kernels: the sparse product with the PageRank update
// fused into its epilogue (by default the sliced sweep slice_spmv, else a
// merge-path kernel, with PagerankEpi) and the split-row / reduction kernel
// (split_rows). A third, normally idle, kernel computes the exact L1 change
// when the fused estimate is too close to the tolerance.
//
// Normalisation is folded into the next sweep. The device stores the
// unnormalised iterate y_k and z_k = y_k / out (0 for dangling nodes); with
// T_k = sum(y_k) the normalised iterate is x_k = y_k / T_k, and one sweep
// computes, for every row i,
//     u_i = d ((A z_k)_i / T_k + (D_k / T_k) jump_i) + (1 - d) p_i
// which is the reference's y_i before its division by `total` (D_k is the
// dangling mass of y_k). The L1 change sum |u_i / T_{k+1} - x_k,i| needs
// T_{k+1}, known only after the sweep; the sweep accumulates
// sum |u_i - x_k,i| instead, which differs from it by at most |1 - T_{k+1}|
// (T is 1 up to rounding since the transition matrix is column
// stochastic). When the estimate is within that bound of the tolerance, the
// exact change is computed by pr_exact_change before deciding.
//
// Mixed precision runs the same trajectory: FP32 sweeps (FP32 arc values,
// iterate and row sums; FP64 reductions) from the uniform start, then one
// FP64 anchor sweep and refinement sweeps (RefineEpi) until the reference's
// stopping rule holds in FP64. The FP32 phase ends when its change falls
// below max(tol * switch_factor, switch_floor): the FP32 perturbation of the
// trajectory (about 1e-7 in L1) then decays over the remaining sweeps by the
// same factor as the change, to well below the tolerance.
#include <algorithm>
#include <cfloat>
#include <map>
#include <mutex>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "bulk.cuh"
#include "pagerank.cuh"

namespace knb {

// ======================================================================= epilogue
template <class VT, bool PV, bool JU, bool EXACT>
struct PagerankEpi {
  static constexpr int NACC = 3;
  static constexpr bool SUMS = true;  // total, dangling mass, change
  const VT* y_old;
  VT* y_new;
  VT* z_new;
  const VT* inv_out;
  const double* p;  // personalization (rescaled), when PV
  double d;
  double pu;        // 1 / n
  VT c_it = 0, c_dt = 0;

  __device__ __forceinline__ void prepare(const IterState* st) {
    c_it = (VT)st->inv_total;
    c_dt = (VT)st->dterm;
  }
  static __device__ __forceinline__ void init(double* a) { a[0] = a[1] = a[2] = 0.0; }
  static __device__ __forceinline__ double identity(int) { return 0.0; }
  static __device__ __forceinline__ double combine(int, double a, double b) { return a + b; }
  static __device__ __forceinline__ double warp_combine(int, double v) { return warp_sum(v); }

  // The per-node inputs of row g's update, loaded apart from it so a sweep
  // can issue these loads before the row sum is ready (fetch, then row_in).
  struct In {
    VT yo, io, pg;
  };
  __device__ __forceinline__ In fetch(uint32_t g) const {
    return {y_old[g], inv_out[g], PV ? (VT)p[g] : (VT)pu};
  }
  __device__ __forceinline__ void row_in(uint32_t g, VT s, const In& in, double* a) const {
    const VT pg = in.pg;
    const VT jg = JU ? (VT)pu : pg;
    const VT u = (VT)d * (s * c_it + c_dt * jg) + (VT)(1.0 - d) * pg;
    const VT xo = in.yo * c_it;
    const VT io = in.io;
    y_new[g] = u;
    z_new[g] = u * io;
    a[0] += (double)u;
    if (io == VT(0)) a[1] += (double)u;
    a[2] += fabs((double)u - (double)xo);
  }
  __device__ __forceinline__ void row(uint32_t g, VT s, double* a) const {
    row_in(g, s, fetch(g), a);
  }

  __device__ void finish(IterState* st, const double* tot) const {
    const double T = tot[0], D = tot[1], ch = tot[2];
    st->prev_inv_total = st->inv_total;
    st->total = T;
    st->dang = D;
    st->change = ch;
    st->inv_total = 1.0 / T;
    st->dterm = D / T;
    st->iter += 1;
    bool amb = false;
    if (EXACT) {
      double slack = 2.0 * fabs(1.0 - T) + 64.0 * DBL_EPSILON * fmax(ch, st->tol);
      st->slack = slack;
      amb = fabs(ch - st->tol) <= slack;
    }
    if (amb) st->ambiguous = 1;
    else if (ch <= st->tol) st->converged = 1;
    else if (st->iter >= st->max_iter) st->stopped = 1;
  }
};

// Refinement sweeps of the mixed path. After the FP32 phase one FP64
// "anchor" sweep fixes y_ref (its input iterate) and keeps the row sums
// s_ref = A (y_ref / out); every later iterate is held as y = y_ref + e with
// e in FP32, and a refinement sweep gathers z_e = e / out in FP32 (FP32
// arc values, FP32 accumulation) and forms s = s_ref + A z_e in FP64. The
// update, the sums and the stopping rule are those of the FP64 sweep
// (PagerankEpi<double>), on the same trajectory: the FP32 rounding now
// applies to e, which is about 1e-5 of y once the FP32 phase has ended, so
// each sweep perturbs the iterate by about 1e-12 instead of 1e-7.
// ANCHOR: the FP64 sweep that computes s_ref (row sums of the FP64 z).
template <class VT, bool ANCHOR, bool PV, bool JU, bool EXACT>
struct RefineEpi {
  static constexpr int NACC = 3;
  static constexpr bool SUMS = true;
  const double* y_ref;
  double* s_ref;        // written by the anchor sweep, read by refinement sweeps
  const float* e_old;   // refinement sweeps: e of the input iterate
  float* e_new;
  float* z_new;         // e_new / out in FP32 (0 for dangling nodes)
  const float* inv_out;
  const double* p;
  double d;
  double pu;
  double c_it = 0, c_dt = 0;

  __device__ __forceinline__ void prepare(const IterState* st) {
    c_it = st->inv_total;
    c_dt = st->dterm;
  }
  static __device__ __forceinline__ void init(double* a) { a[0] = a[1] = a[2] = 0.0; }
  static __device__ __forceinline__ double identity(int) { return 0.0; }
  static __device__ __forceinline__ double combine(int, double a, double b) { return a + b; }
  static __device__ __forceinline__ double warp_combine(int, double v) { return warp_sum(v); }

  // The per-node inputs of row g's update (see PagerankEpi::fetch).
  struct In {
    double sr, yr, pg;
    float eo, io;
  };
  __device__ __forceinline__ In fetch(uint32_t g) const {
    In in;
    in.sr = ANCHOR ? 0.0 : s_ref[g];
    in.yr = y_ref[g];
    in.pg = PV ? p[g] : pu;
    in.eo = ANCHOR ? 0.0f : e_old[g];
    in.io = inv_out[g];
    return in;
  }
  __device__ __forceinline__ void row_in(uint32_t g, VT s_in, const In& in, double* a) const {
    double s;
    if constexpr (ANCHOR) {
      s = (double)s_in;
      s_ref[g] = s;
    } else {
      s = in.sr + (double)s_in;
    }
    const double pg = in.pg;
    const double jg = JU ? pu : pg;
    const double u = d * (s * c_it + c_dt * jg) + (1.0 - d) * pg;
    const double yr = in.yr;
    const double yo = ANCHOR ? yr : yr + (double)in.eo;
    const float en = (float)(u - yr);
    const double us = yr + (double)en;  // the iterate as stored
    const float io = in.io;
    e_new[g] = en;
    z_new[g] = en * io;
    a[0] += us;
    if (io == 0.0f) a[1] += us;
    a[2] += fabs(us - yo * c_it);
  }
  __device__ __forceinline__ void row(uint32_t g, VT s_in, double* a) const {
    row_in(g, s_in, fetch(g), a);
  }

  __device__ void finish(IterState* st, const double* tot) const {
    PagerankEpi<double, PV, JU, EXACT> base;
    base.finish(st, tot);
  }
};

// ======================================================================= vertex kernels
constexpr int VT_THREADS = 256;

// Last-CTA fixed-order sum of `k` partial arrays of `nb` blocks each.
__device__ __forceinline__ bool last_block(unsigned int* ticket) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last) __threadfence();
  return last;
}

template <int K>
__device__ __forceinline__ void reduce_parts(const double* part, uint32_t nb, double* out,
                                             double* scratch) {
  const volatile double* p = part;
  for (int s = 0; s < K; ++s) {
    double a = 0;
    for (uint32_t q = threadIdx.x; q < nb; q += blockDim.x) a += p[(size_t)q * K + s];
    a = block_sum(a, scratch);
    out[s] = a;
  }
}

// x0 = 1/n, z0 = x0 / out, D0 = dangling mass (spectral.rs:248-259).
template <class VT>
__global__ void pr_init(VT* __restrict__ y, VT* __restrict__ z, const VT* __restrict__ inv_out,
                        uint32_t n, double* __restrict__ part, IterState* st) {
  __shared__ double sh[VT_THREADS / 32];
  const VT x0 = (VT)(1.0 / (double)n);
  double dang = 0, tot = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    VT io = inv_out[i];
    y[i] = x0;
    z[i] = x0 * io;
    tot += (double)x0;
    if (io == VT(0)) dang += (double)x0;
  }
  dang = block_sum(dang, sh);
  tot = block_sum(tot, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x * 2] = tot;
    part[blockIdx.x * 2 + 1] = dang;
  }
  if (!last_block(&st->ticket)) return;
  double r[2];
  reduce_parts<2>(part, gridDim.x, r, sh);
  if (threadIdx.x == 0) {
    st->inv_total = 1.0;
    st->dterm = r[1];
    st->total = r[0];
    st->prev_inv_total = 1.0;
    st->ticket = 0;
  }
}

// Exact L1 change sum |y_new / T - y_old * prev_inv_total| when the fused
// estimate cannot decide (see the file comment).
__global__ void pr_exact_change(const double* __restrict__ y_old, const double* __restrict__ y_new,
                                uint32_t n, double* __restrict__ part, IterState* st) {
  if (!st->ambiguous || st->converged || st->stopped) return;
  __shared__ double sh[VT_THREADS / 32];
  const double T = st->total, ip = st->prev_inv_total;
  double a = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    a += fabs(y_new[i] / T - y_old[i] * ip);
  a = block_sum(a, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = a;
  if (!last_block(&st->ticket2)) return;
  double r[1];
  reduce_parts<1>(part, gridDim.x, r, sh);
  if (threadIdx.x == 0) {
    st->change = r[0];
    st->ambiguous = 0;
    if (r[0] <= st->tol) st->converged = 1;
    else if (st->iter >= st->max_iter) st->stopped = 1;
    st->ticket2 = 0;
  }
}

// The exact change for refinement sweeps, whose iterates are y_ref + e
// (e_old null: the anchor sweep, whose input iterate is y_ref itself).
__global__ void pr_exact_change_ref(const double* __restrict__ y_ref,
                                    const float* __restrict__ e_old,
                                    const float* __restrict__ e_new, uint32_t n,
                                    double* __restrict__ part, IterState* st) {
  if (!st->ambiguous || st->converged || st->stopped) return;
  __shared__ double sh[VT_THREADS / 32];
  const double T = st->total, ip = st->prev_inv_total;
  double a = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double yr = y_ref[i];
    const double yo = e_old ? yr + (double)e_old[i] : yr;
    a += fabs((yr + (double)e_new[i]) / T - yo * ip);
  }
  a = block_sum(a, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = a;
  if (!last_block(&st->ticket2)) return;
  double r[1];
  reduce_parts<1>(part, gridDim.x, r, sh);
  if (threadIdx.x == 0) {
    st->change = r[0];
    st->ambiguous = 0;
    if (r[0] <= st->tol) st->converged = 1;
    else if (st->iter >= st->max_iter) st->stopped = 1;
    st->ticket2 = 0;
  }
}

// out = (y_ref + e) / T in the caller's node order.
__global__ void pr_output_ref(const double* __restrict__ y_ref, const float* __restrict__ e,
                              const IterState* __restrict__ st, uint32_t n,
                              const uint32_t* __restrict__ iperm, double* __restrict__ out) {
  const double T = st->total;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t k = iperm ? iperm[i] : i;
    out[i] = (y_ref[k] + (double)e[k]) / T;
  }
}

// FP32 -> FP64 hand-over: y64 = y32 / T32, z64 = y64 / out, new scalars.
__global__ void pr_switch(const float* __restrict__ y32, const IterState* __restrict__ st32,
                          double* __restrict__ y64, double* __restrict__ z64,
                          const double* __restrict__ inv_out, uint32_t n,
                          double* __restrict__ part, IterState* st) {
  __shared__ double sh[VT_THREADS / 32];
  const double it = st32->inv_total;
  double tot = 0, dang = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double y = (double)y32[i] * it;
    double io = inv_out[i];
    y64[i] = y;
    z64[i] = y * io;
    tot += y;
    if (io == 0.0) dang += y;
  }
  tot = block_sum(tot, sh);
  dang = block_sum(dang, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x * 2] = tot;
    part[blockIdx.x * 2 + 1] = dang;
  }
  if (!last_block(&st->ticket)) return;
  double r[2];
  reduce_parts<2>(part, gridDim.x, r, sh);
  if (threadIdx.x == 0) {
    st->total = r[0];
    st->inv_total = 1.0 / r[0];
    st->prev_inv_total = st->inv_total;
    st->dterm = r[1] / r[0];
    st->ticket = 0;
  }
}

// out = y / T (spectral.rs:268-270), in FP64, in the caller's node order
// (iperm maps a node to its number in a relabelled operator, or is null).
template <class VT>
__global__ void pr_output(const VT* __restrict__ y, const IterState* __restrict__ st, uint32_t n,
                          const uint32_t* __restrict__ iperm, double* __restrict__ out) {
  const double T = st->total;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = (double)y[iperm ? iperm[i] : i] / T;
}

__global__ void permute_in(const double* __restrict__ in, const uint32_t* __restrict__ perm,
                           uint32_t n, double* __restrict__ out) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[k] = in[perm[k]];
}

// Personalization checks and rescaling to sum 1 (spectral.rs:284-304): the
// first pass finds any value that is not finite or negative and sums the
// rest in a fixed order; the second divides by the sum.
__global__ void pers_check(const double* __restrict__ p, uint32_t n, double* __restrict__ part,
                           IterState* st) {
  __shared__ double sh[VT_THREADS / 32];
  double a = 0, bad = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = p[i];
    if (!isfinite(v) || v < 0.0) bad = 1;
    else a += v;
  }
  a = block_sum(a, sh);
  bad = block_sum(bad, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x * 2] = a;
    part[blockIdx.x * 2 + 1] = bad;
  }
  if (!last_block(&st->ticket)) return;
  double r[2];
  reduce_parts<2>(part, gridDim.x, r, sh);
  if (threadIdx.x == 0) {
    st->total = r[0];
    st->stopped = r[1] > 0 ? 1 : 0;
    st->ticket = 0;
  }
}

__global__ void pers_scale(double* __restrict__ p, uint32_t n, const IterState* __restrict__ st) {
  const double sum = st->total;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    p[i] = p[i] / sum;
}

static void normalize_personalization(double* p, uint32_t n, double* part, IterState* st,
                                      IterState* hst, cudaStream_t s) {
  const unsigned gv = grid_for(n, VT_THREADS, 1184);
  KNB_CUDA(cudaMemsetAsync(st, 0, sizeof(IterState), s));
  pers_check<<<gv, VT_THREADS, 0, s>>>(p, n, part, st);
  KNB_LAUNCH("pers_check");
  KNB_CUDA(cudaMemcpyAsync(hst, st, sizeof(IterState), cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  if (hst->stopped) throw Error("the personalization vector must hold finite, nonnegative values");
  if (!(hst->total > 0.0)) throw Error("the personalization vector must have a positive sum");
  pers_scale<<<gv, VT_THREADS, 0, s>>>(p, n, st);
  KNB_LAUNCH("pers_scale");
}

void normalize_personalization_device(double* p, uint32_t n, cudaStream_t s) {
  const unsigned gv = grid_for(n, VT_THREADS, 1184);
  DevBuf<double> part((size_t)gv * 2 + 8);
  DevBuf<IterState> st(1);
  IterState* hst = nullptr;
  KNB_CUDA(cudaMallocHost(&hst, sizeof(IterState)));
  try {
    normalize_personalization(p, n, part.get(), st.get(), hst, s);
  } catch (...) {
    cudaFreeHost(hst);
    throw;
  }
  KNB_CUDA(cudaFreeHost(hst));
}

// Scratch of PageRank solves on one operator, kept between calls: iterates,
// per-tile partials, carries, states, pinned host state slots and events.
// A solve holds `mu` while it runs, so concurrent calls on one operator take
// turns instead of sharing buffers.
struct PrWorkspace : Workspace {
  std::mutex mu;
  uint32_t n = 0, nt = 0;
  DevBuf<double> y64[2], z64[2], carry64, head64, pvec, ptmp, dout, part1, part2, part3;
  DevBuf<float> y32[2], z32[2], carry32, head32;
  DevBuf<IterState> st;        // 0: FP32 phase, 1: FP64 phase, 2: personalization
  IterState* hstate = nullptr;  // pinned, 3 slots
  cudaEvent_t t0 = nullptr, t1 = nullptr, done[2] = {nullptr, nullptr};
  cudaEvent_t a0 = nullptr, a1 = nullptr;  // anchor-sweep timing
  std::vector<cudaEvent_t> pool;  // sweep-timing events

  ~PrWorkspace() override {
    if (hstate) cudaFreeHost(hstate);
    for (cudaEvent_t e : {t0, t1, done[0], done[1], a0, a1})
      if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : pool) cudaEventDestroy(e);
  }
  void ensure(uint32_t nn, uint32_t ntiles, bool need32, bool need64, bool need_p) {
    if (!hstate) {
      KNB_CUDA(cudaMallocHost(&hstate, 3 * sizeof(IterState)));
      KNB_CUDA(cudaEventCreate(&t0));
      KNB_CUDA(cudaEventCreate(&t1));
      KNB_CUDA(cudaEventCreate(&a0));
      KNB_CUDA(cudaEventCreate(&a1));
      KNB_CUDA(cudaEventCreateWithFlags(&done[0], cudaEventDisableTiming));
      KNB_CUDA(cudaEventCreateWithFlags(&done[1], cudaEventDisableTiming));
      st.alloc(3);
    }
    const unsigned gv = grid_for(nn, VT_THREADS, 1184);
    if (n != nn) {
      n = nn;
      for (int k = 0; k < 2; ++k) {
        y32[k].release(); z32[k].release(); y64[k].release(); z64[k].release();
      }
      pvec.release(); ptmp.release(); dout.release();
      part3.alloc((size_t)gv * 2 + 8);
      part2.alloc((size_t)SPLIT_CTAS * 3 + 8);
    }
    if (nt < ntiles) {
      nt = ntiles;
      part1.alloc((size_t)nt * 3 + 8);
      carry32.release(); head32.release(); carry64.release(); head64.release();
    }
    if (need32 && !y32[0].p) {
      for (int k = 0; k < 2; ++k) { y32[k].alloc(n); z32[k].alloc(n); }
    }
    if (need32 && !carry32.p) { carry32.alloc(nt + 1); head32.alloc(nt + 1); }
    if (need64 && !y64[0].p) {
      for (int k = 0; k < 2; ++k) { y64[k].alloc(n); z64[k].alloc(n); }
    }
    if (need64 && !carry64.p) { carry64.alloc(nt + 1); head64.alloc(nt + 1); }
    if (need_p && !pvec.p) { pvec.alloc(n); ptmp.alloc(n); }
  }
  cudaEvent_t timing_event(size_t k) {
    while (pool.size() <= k) {
      cudaEvent_t e;
      KNB_CUDA(cudaEventCreate(&e));
      pool.push_back(e);
    }
    return pool[k];
  }
};

// ======================================================================= sweeps
struct SweepBuffers {
  OpView<double> v64;
  OpView<float> v32;
  void* y[2];
  void* z[2];
  const void* inv_out;
  const double* p;
  void* carry;
  void* head;
  double* part1;
  double* part2;
  double* part3;
  IterState* st;
  const double* y_ref = nullptr;  // refinement sweeps: the anchor iterate (FP64)
  double* s_ref = nullptr;        //   and its row sums
  const SlicedOp* so = nullptr;   // the sliced layout (slice variants)
};

enum SweepVariant : int {
  VAR_CTA = 1, VAR_WARP = 2, VAR_WARP4 = 3, VAR_WARP16 = 4, VAR_WARPNA = 5,
  VAR_HOT = 6,    // hot-node cache, one CTA of 32 warps per SM
  VAR_HOT16 = 7,  // hot-node cache, one CTA of 16 warps per SM
  VAR_WARPL1 = 8, // 16 warps per CTA; only gathers of the most gathered columns allocate in L1
  VAR_SLICE = 9,    // sliced layout (slice.cuh), 48 resident warps per SM
  VAR_SLICE64 = 10, // sliced layout, 64 resident warps per SM
  VAR_SLICEH = 11,  // sliced layout, one 32-warp CTA per SM, most gathered values in shared memory
  VAR_SLICEB = 12,  // sliced layout, arc streams staged in shared memory by bulk copies
};
static bool slice_variant(int var) { return var >= VAR_SLICE && var <= VAR_SLICEB; }
static bool slice64_variant(int var) { return var == VAR_SLICE64; }

// Columns whose gathers allocate in L1 (FP32 values): the tuned choice of the
// solve running on this thread, else the process-wide tuning (-1: each
// kernel's default).
static thread_local int64_t g_hot_override = -1;
static int64_t hot_setting() { return g_hot_override >= 0 ? g_hot_override : tuning().hot_nodes; }
struct HotOverride {
  int64_t saved;
  explicit HotOverride(int64_t v) : saved(g_hot_override) { g_hot_override = v; }
  ~HotOverride() { g_hot_override = saved; }
};

// SM count and the largest dynamic shared memory a CTA may opt into, per
// device (queried once).
struct DeviceLimits {
  int sms = 0;
  int smem_optin = 0;
};
static DeviceLimits device_limits() {
  static std::mutex mu;
  static std::map<int, DeviceLimits> cache;
  int dev = 0;
  KNB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(dev);
  if (it != cache.end()) return it->second;
  DeviceLimits d;
  KNB_CUDA(cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev));
  KNB_CUDA(cudaDeviceGetAttribute(&d.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cache[dev] = d;
  return d;
}

// Nodes the hot-node sweep keeps in shared memory: as many as fit beside
// the warp buffers, at most n (and at most the tuning cap), in whole
// 16-byte vectors.
template <class VT>
static uint32_t hot_nodes(uint32_t n, size_t warp_bytes, int smem_optin) {
  const size_t room = (size_t)smem_optin > warp_bytes ? (size_t)smem_optin - warp_bytes : 0;
  uint64_t hn = std::min<uint64_t>(room / sizeof(VT), n);
  if (tuning().hot_nodes >= 0) hn = std::min<uint64_t>(hn, (uint64_t)tuning().hot_nodes);
  hn -= hn % (16 / sizeof(VT));
  return (uint32_t)hn;
}

// CTAs of a sliced sweep that fit on the device at once (per device and
// shared-memory size).
template <class VT, class MT, class Epi, int U, int WPB, int MINB, int GNA>
static unsigned slice_grid(size_t smem) {
  static std::mutex mu;
  static std::map<std::pair<int, size_t>, unsigned> grids;
  int dev = 0;
  KNB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(dev, smem);
  auto it = grids.find(key);
  if (it != grids.end()) return it->second;
  int per_sm = 0;
  KNB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &per_sm, slice_spmv<VT, MT, Epi, U, WPB, MINB, GNA>, WPB * 32, smem));
  const unsigned g = (unsigned)std::max(1, per_sm) * (unsigned)device_limits().sms;
  grids[key] = g;
  return g;
}

// Sliced sweeps: a persistent grid of the CTAs that fit at once. Only
// gathers of the most gathered columns allocate in L1: 49,152 FP32 values
// (192 KB) by default, as many bytes of FP64 values (measured on R-MAT 24:
// no L1 allocation at all makes the FP32 sweep 1.36 ms instead of 0.83 ms;
// 24,576, 98,304 or every column 0.86-0.88 ms). Without a shared-memory
// tier the kernel asks for the smallest carveout, so L1 keeps the SM's whole
// 256 KB; with one (HOT), one CTA per SM keeps the first smem_n values of
// the iterate in shared memory and the carveout is what that needs.
template <class VT, class MT, class Epi, int U, int MINB, bool HOT>
static unsigned launch_slice(const SlicedOp& so, const VT* x, const Epi& e, VT* carry, VT* head,
                             double* part1, IterState* st, cudaStream_t s) {
  constexpr int GNA = 2;
  constexpr int WPB = HOT ? SLICE_HOT_WPB : SLICE_WPB;
  auto fnp = slice_spmv<VT, MT, Epi, U, WPB, HOT ? 1 : MINB, GNA>;
  uint32_t smem_n = 0;
  if constexpr (HOT) {
    const int64_t want = tuning().smem_hot >= 0 ? tuning().smem_hot : 32768;
    const uint64_t cap = (uint64_t)(device_limits().smem_optin - 1024) / sizeof(VT);
    uint64_t hn = std::min<uint64_t>({(uint64_t)want * 4 / sizeof(VT), cap, (uint64_t)so.n});
    hn -= hn % (16 / sizeof(VT));
    smem_n = (uint32_t)hn;
  }
  const size_t smem = (size_t)smem_n * sizeof(VT);
  if (smem) set_func_attr((const void*)fnp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int carve = smem ? std::min(100, (int)((smem + 1024) * 100 / 233472) + 1) : 0;
  set_func_attr((const void*)fnp, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
  const unsigned grid = slice_grid<VT, MT, Epi, U, WPB, HOT ? 1 : MINB, GNA>(smem);
  const uint64_t hot32 = hot_setting() >= 0 ? (uint64_t)hot_setting() : 49152u;
  const uint32_t l1_hot = (uint32_t)std::min<uint64_t>(hot32 * 4 / sizeof(VT), 0xFFFFFFFFull);
  fnp<<<grid, WPB * 32, smem, s>>>(so.view<MT>(), x, e, carry, head, part1, st, l1_hot, smem_n);
  return grid * WPB;
}

// Bulk-staged sliced sweeps (bulk.cuh): U arc positions per chunk, S stages
// per warp (4 for U = 4, 3 for U = 8), 8 warps per CTA. The carveout asks
// for the shared memory of `ctas` CTAs per SM (default 4: 32 warps and 135
// KB of rings for FP32 values, the rest of the SM's 256 KB left to L1); the
// grid is every CTA that fits at once.
constexpr int BULK_WPB = 8;
template <class VT, class MT, class Epi, int U>
static unsigned launch_slice_bulk(const SlicedOp& so, const VT* x, const Epi& e, VT* carry,
                                  VT* head, double* part1, IterState* st, cudaStream_t s) {
  constexpr int GNA = 2;
  constexpr int S = U >= 8 ? 3 : 4;
  auto fnp = slice_bulk_spmv<VT, MT, Epi, U, S, BULK_WPB, 4, GNA>;
  const size_t smem = (size_t)BULK_WPB * bulk_ring_bytes<MT, U, S>();
  const int ctas = tuning().bulk_ctas > 0 ? tuning().bulk_ctas : 4;
  set_func_attr((const void*)fnp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const int carve = std::min(100, (int)(((smem + 1024) * ctas * 100 + 233471) / 233472));
  set_func_attr((const void*)fnp, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
  static std::mutex mu;
  static std::map<std::tuple<int, const void*, int>, unsigned> grids;
  int dev = 0;
  KNB_CUDA(cudaGetDevice(&dev));
  unsigned grid = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_tuple(dev, (const void*)fnp, ctas);
    auto it = grids.find(key);
    if (it == grids.end()) {
      int per_sm = 0;
      KNB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fnp, BULK_WPB * 32, smem));
      per_sm = std::max(1, std::min(per_sm, ctas));
      it = grids.emplace(key, (unsigned)per_sm * (unsigned)device_limits().sms).first;
    }
    grid = it->second;
  }
  const uint64_t hot32 = hot_setting() >= 0 ? (uint64_t)hot_setting() : 49152u;
  const uint32_t l1_hot = (uint32_t)std::min<uint64_t>(hot32 * 4 / sizeof(VT), 0xFFFFFFFFull);
  const uint32_t skip =
      tuning().bulk_skip_chunk >= 0 ? (uint32_t)tuning().bulk_skip_chunk : BULK_NO_SKIP;
  fnp<<<grid, BULK_WPB * 32, smem, s>>>(so.view<MT>(), x, e, carry, head, part1, st, l1_hot,
                                        skip);
  return grid * BULK_WPB;
}

// One sweep with epilogue `e`: the sweep kernel of variant VAR gathering x
// (sliced, bulk-staged or merge-path), then the split-row kernel, whose CTAs
// also reduce the epilogue's per-tile or per-warp scalars and whose last CTA
// decides convergence.
template <class VT, class MT, class Epi, int VAR, int IPT>
static void launch_spmv(const Operator& op, const Partition& P, const OpView<MT>& v,
                        const VT* x, const Epi& e, VT* carry, VT* head, double* part1,
                        double* part2, IterState* st, cudaStream_t s, unsigned g2,
                        cudaEvent_t ev0, cudaEvent_t ev1, const SlicedOp* so = nullptr) {
  if (ev0) KNB_CUDA(cudaEventRecord(ev0, s));
  uint32_t npart = P.ntiles;  // partials the sweep leaves for split_rows
  if constexpr (VAR >= VAR_SLICE && VAR <= VAR_SLICEB) {
    if constexpr (VAR == VAR_SLICEB) {
      npart = launch_slice_bulk<VT, MT, Epi, IPT>(*so, x, e, carry, head, part1, st, s);
      KNB_LAUNCH("slice_bulk_spmv");
    } else {
      constexpr int MINB = VAR == VAR_SLICE64 ? 8 : 6;
      npart = launch_slice<VT, MT, Epi, IPT, MINB, VAR == VAR_SLICEH>(*so, x, e, carry, head,
                                                                      part1, st, s);
      KNB_LAUNCH("slice_spmv");
    }
    if (ev1) KNB_CUDA(cudaEventRecord(ev1, s));
    split_rows<VT, Epi><<<g2, SPMV_THREADS, 0, s>>>(so->split.get(), so->nsplit, so->nshort,
                                                     carry, head, e, part1, npart, part2, st);
    KNB_LAUNCH("split_rows");
    return;
  } else if constexpr (VAR == VAR_HOT || VAR == VAR_HOT16) {
    constexpr int WPB = VAR == VAR_HOT ? 32 : 16;
    constexpr size_t wbytes = hot_warp_smem_bytes<VT, IPT, WPB>();
    const DeviceLimits lim = device_limits();
    const uint32_t hn = hot_nodes<VT>(op.n, wbytes, lim.smem_optin);
    const size_t smem = wbytes + (size_t)hn * sizeof(VT);
    auto fnp = hot_spmv<VT, MT, Epi, IPT, WPB>;
    static std::mutex attr_mu;
    static std::map<int, size_t> attr_set;  // per device: the largest size allowed so far
    {
      int dev = 0;
      KNB_CUDA(cudaGetDevice(&dev));
      std::lock_guard<std::mutex> lock(attr_mu);
      size_t& allowed = attr_set[dev];
      if (smem > allowed) {
        KNB_CUDA(cudaFuncSetAttribute(fnp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        allowed = smem;
      }
    }
    const unsigned grid = (unsigned)std::max(1, std::min<int>(lim.sms, (P.ntiles + WPB - 1) / WPB));
    npart = std::min<uint32_t>(P.ntiles, grid * WPB);
    hot_spmv<VT, MT, Epi, IPT, WPB><<<grid, WPB * 32, smem, s>>>(
        v, x, hn, e, P.coords.get(), P.ntiles, carry, head,
        part1, st);
  } else if constexpr (VAR == VAR_CTA) {
    constexpr size_t smem = tile_smem_bytes<VT, IPT>();
    set_func_attr((const void*)tile_spmv<VT, MT, Epi, IPT>,
                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    tile_spmv<VT, MT, Epi, IPT><<<P.ntiles, SPMV_THREADS, smem, s>>>(
        v, x, e, P.coords.get(), carry, head, part1, st);
  } else {
    constexpr int WPB = VAR == VAR_WARP4 ? 4 : (VAR == VAR_WARP16 || VAR == VAR_WARPL1) ? 16 : 8;
    constexpr int GNA = VAR == VAR_WARPNA ? 1 : VAR == VAR_WARPL1 ? 2 : 0;
    constexpr size_t smem = warp_smem_bytes<VT, IPT, WPB>();
    auto fnp = warp_spmv<VT, MT, Epi, IPT, WPB, GNA>;
    set_func_attr((const void*)fnp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // Shared-memory carveout: by default just enough for the CTAs the kernel
    // is built to keep resident (each with its dynamic shared memory and the
    // 1 KB the driver reserves), as a percentage of the 228 KB an SM has; the
    // driver rounds the hint up to the next configuration it supports, and
    // the rest of the SM's 256 KB stays L1. Left to itself the driver picks a
    // larger configuration (132 KB for the FP32 sweep's 78 KB), 2-3% slower.
    const int carve =
        tuning().carveout >= 0 ? tuning().carveout : warp_fit_carveout<VT, IPT, WPB>();
    set_func_attr((const void*)fnp, cudaFuncAttributePreferredSharedMemoryCarveout, carve);
    unsigned grid = (P.ntiles + WPB - 1) / WPB;
    if (tuning().persistent) {
      // the CTAs that fit on the GPU at once, each warp looping over tiles
      static std::mutex occ_mu;
      static std::map<std::pair<int, int>, int> occ;  // (device, carveout) -> CTAs per SM
      int dev = 0;
      KNB_CUDA(cudaGetDevice(&dev));
      int per_sm = 0;
      {
        std::lock_guard<std::mutex> lock(occ_mu);
        auto key = std::make_pair(dev, carve);
        auto it = occ.find(key);
        if (it == occ.end()) {
          KNB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fnp, WPB * 32, smem));
          occ[key] = per_sm;
        } else {
          per_sm = it->second;
        }
      }
      const unsigned cap = (unsigned)std::max(1, per_sm) * (unsigned)device_limits().sms;
      grid = std::min(grid, cap);
    }
    // L1-allocating gathers only below this column (GNA 2)
    const uint32_t l1_hot = hot_setting() >= 0 ? (uint32_t)std::min<int64_t>(
                                                     hot_setting(), 0xFFFFFFFFll)
                                               : 24576u;
    npart = std::min<uint32_t>(P.ntiles, grid * WPB);
    warp_spmv<VT, MT, Epi, IPT, WPB, GNA><<<grid, WPB * 32, smem, s>>>(
        v, x, e, P.coords.get(), P.ntiles, carry, head,
        part1, st, l1_hot);
  }
  KNB_LAUNCH("sweep");
  if (ev1) KNB_CUDA(cudaEventRecord(ev1, s));
  split_rows<VT, Epi><<<g2, SPMV_THREADS, 0, s>>>(P.split.get(), P.nsplit, P.nshort,
                                                   carry, head, e,
                                                   part1, npart, part2, st);
  KNB_LAUNCH("split_rows");
}

template <class VT, class MT, bool PV, bool JU, bool EXACT, int VAR, int IPT>
static void launch_sweep(const Operator& op, const Partition& P, const SweepBuffers& B, int buf,
                         double d, cudaStream_t s, unsigned g2, cudaEvent_t ev0, cudaEvent_t ev1) {
  using Epi = PagerankEpi<VT, PV, JU, EXACT>;
  Epi e;
  e.y_old = (const VT*)B.y[buf];
  e.y_new = (VT*)B.y[1 - buf];
  e.z_new = (VT*)B.z[1 - buf];
  e.inv_out = (const VT*)B.inv_out;
  e.p = B.p;
  e.d = d;
  e.pu = 1.0 / (double)op.n;
  OpView<MT> v;
  if constexpr (sizeof(MT) == 8) v = B.v64; else v = B.v32;
  launch_spmv<VT, MT, Epi, VAR, IPT>(op, P, v, (const VT*)B.z[buf], e, (VT*)B.carry,
                                     (VT*)B.head, B.part1, B.part2, B.st, s, g2, ev0, ev1, B.so);
  if (EXACT) {
    pr_exact_change<<<grid_for(op.n, VT_THREADS, 1184), VT_THREADS, 0, s>>>(
        (const double*)B.y[buf], (const double*)B.y[1 - buf], op.n, B.part3, B.st);
    KNB_LAUNCH("pr_exact_change");
  }
}

using SweepFn = void (*)(const Operator&, const Partition&, const SweepBuffers&, int, double,
                         cudaStream_t, unsigned, cudaEvent_t, cudaEvent_t);

template <class VT, class MT, bool EXACT, int VAR, int IPT>
static SweepFn pick_pv(bool pv, bool ju) {
  if (!pv) return launch_sweep<VT, MT, false, true, EXACT, VAR, IPT>;
  if (ju) return launch_sweep<VT, MT, true, true, EXACT, VAR, IPT>;
  return launch_sweep<VT, MT, true, false, EXACT, VAR, IPT>;
}

template <class VT, class MT, bool EXACT, int VAR>
static SweepFn pick_warp_ipt(int ipt, bool pv, bool ju) {
  switch (ipt) {
    case 4: return pick_pv<VT, MT, EXACT, VAR, 4>(pv, ju);
    case 16: return pick_pv<VT, MT, EXACT, VAR, 16>(pv, ju);
    default: return pick_pv<VT, MT, EXACT, VAR, 8>(pv, ju);
  }
}

template <class VT, class MT, bool EXACT>
static SweepFn pick_kernel(int var, int ipt, bool pv, bool ju) {
  switch (var) {
    case VAR_CTA:
      return ipt == 4 ? pick_pv<VT, MT, EXACT, VAR_CTA, 4>(pv, ju)
                      : pick_pv<VT, MT, EXACT, VAR_CTA, 8>(pv, ju);
    case VAR_WARP4: return pick_warp_ipt<VT, MT, EXACT, VAR_WARP4>(ipt, pv, ju);
    case VAR_WARP16: return pick_warp_ipt<VT, MT, EXACT, VAR_WARP16>(ipt, pv, ju);
    case VAR_WARPNA: return pick_warp_ipt<VT, MT, EXACT, VAR_WARPNA>(ipt, pv, ju);
    case VAR_HOT: return pick_warp_ipt<VT, MT, EXACT, VAR_HOT>(ipt, pv, ju);
    case VAR_HOT16: return pick_warp_ipt<VT, MT, EXACT, VAR_HOT16>(ipt, pv, ju);
    case VAR_WARPL1: return pick_warp_ipt<VT, MT, EXACT, VAR_WARPL1>(ipt, pv, ju);
    case VAR_SLICE:
      return ipt == 4 ? pick_pv<VT, MT, EXACT, VAR_SLICE, 4>(pv, ju)
                      : pick_pv<VT, MT, EXACT, VAR_SLICE, 8>(pv, ju);
    case VAR_SLICE64: return pick_pv<VT, MT, EXACT, VAR_SLICE64, 4>(pv, ju);
    case VAR_SLICEH:
      return ipt == 4 ? pick_pv<VT, MT, EXACT, VAR_SLICEH, 4>(pv, ju)
                      : pick_pv<VT, MT, EXACT, VAR_SLICEH, 8>(pv, ju);
    case VAR_SLICEB:
      return ipt == 4 ? pick_pv<VT, MT, EXACT, VAR_SLICEB, 4>(pv, ju)
                      : pick_pv<VT, MT, EXACT, VAR_SLICEB, 8>(pv, ju);
    default: return pick_warp_ipt<VT, MT, EXACT, VAR_WARP>(ipt, pv, ju);
  }
}

// ----------------------------------------------------------------------- refinement
// A refinement sweep (RefineEpi): e = B.y[buf] and z_e = B.z[buf] (FP32) in,
// B.y[1 - buf] and B.z[1 - buf] out; FP32 arc values.
template <bool PV, bool JU, int VAR, int IPT>
static void launch_refine(const Operator& op, const Partition& P, const SweepBuffers& B, int buf,
                          double d, cudaStream_t s, unsigned g2, cudaEvent_t ev0,
                          cudaEvent_t ev1) {
  using Epi = RefineEpi<float, false, PV, JU, true>;
  Epi e;
  e.y_ref = B.y_ref;
  e.s_ref = B.s_ref;
  e.e_old = (const float*)B.y[buf];
  e.e_new = (float*)B.y[1 - buf];
  e.z_new = (float*)B.z[1 - buf];
  e.inv_out = (const float*)B.inv_out;
  e.p = B.p;
  e.d = d;
  e.pu = 1.0 / (double)op.n;
  launch_spmv<float, float, Epi, VAR, IPT>(op, P, B.v32, (const float*)B.z[buf], e,
                                           (float*)B.carry, (float*)B.head, B.part1, B.part2,
                                           B.st, s, g2, ev0, ev1, B.so);
  pr_exact_change_ref<<<grid_for(op.n, VT_THREADS, 1184), VT_THREADS, 0, s>>>(
      B.y_ref, (const float*)B.y[buf], (const float*)B.y[1 - buf], op.n, B.part3, B.st);
  KNB_LAUNCH("pr_exact_change_ref");
}

// The anchor sweep: an FP64 sweep gathering z_ref = y_ref / out that keeps
// its row sums in B.s_ref and writes e and z_e of its result to B.y[0] and
// B.z[0]. MT: the arc value type (FP32 when every value is exact in FP32).
template <class MT, bool PV, bool JU, int VAR, int IPT>
static void launch_anchor(const Operator& op, const Partition& P, const SweepBuffers& B,
                          const double* z_ref, double* carry64, double* head64, double d,
                          cudaStream_t s, unsigned g2, cudaEvent_t ev0, cudaEvent_t ev1) {
  using Epi = RefineEpi<double, true, PV, JU, true>;
  Epi e;
  e.y_ref = B.y_ref;
  e.s_ref = B.s_ref;
  e.e_old = nullptr;
  e.e_new = (float*)B.y[0];
  e.z_new = (float*)B.z[0];
  e.inv_out = (const float*)B.inv_out;
  e.p = B.p;
  e.d = d;
  e.pu = 1.0 / (double)op.n;
  OpView<MT> v;
  if constexpr (sizeof(MT) == 8) v = B.v64; else v = B.v32;
  launch_spmv<double, MT, Epi, VAR, IPT>(op, P, v, z_ref, e, carry64, head64, B.part1, B.part2,
                                         B.st, s, g2, ev0, ev1, B.so);
  pr_exact_change_ref<<<grid_for(op.n, VT_THREADS, 1184), VT_THREADS, 0, s>>>(
      B.y_ref, nullptr, (const float*)B.y[0], op.n, B.part3, B.st);
  KNB_LAUNCH("pr_exact_change_ref");
}

using AnchorFn = void (*)(const Operator&, const Partition&, const SweepBuffers&, const double*,
                          double*, double*, double, cudaStream_t, unsigned, cudaEvent_t,
                          cudaEvent_t);

// Refinement and anchor sweeps come in the warp-tile variants (4, 8 or 16
// warps per CTA) with 4 or 8 items per lane; other settings use 16 warps.
template <int VAR, int IPT>
static SweepFn pick_refine_pv(bool pv, bool ju) {
  if (!pv) return launch_refine<false, true, VAR, IPT>;
  if (ju) return launch_refine<true, true, VAR, IPT>;
  return launch_refine<true, false, VAR, IPT>;
}
template <int VAR>
static SweepFn pick_refine_ipt(int ipt, bool pv, bool ju) {
  return ipt == 4 ? pick_refine_pv<VAR, 4>(pv, ju) : pick_refine_pv<VAR, 8>(pv, ju);
}
static SweepFn pick_refine(int var, int ipt, bool pv, bool ju) {
  switch (var) {
    case VAR_SLICE: return pick_refine_pv<VAR_SLICE, 4>(pv, ju);
    case VAR_SLICE64: return pick_refine_pv<VAR_SLICE64, 4>(pv, ju);
    case VAR_SLICEH: return pick_refine_pv<VAR_SLICEH, 4>(pv, ju);
    case VAR_SLICEB: return pick_refine_ipt<VAR_SLICEB>(ipt, pv, ju);
    case VAR_WARP: return pick_refine_ipt<VAR_WARP>(ipt, pv, ju);
    case VAR_WARP4: return pick_refine_ipt<VAR_WARP4>(ipt, pv, ju);
    case VAR_WARPL1: return pick_refine_ipt<VAR_WARPL1>(ipt, pv, ju);
    default: return pick_refine_ipt<VAR_WARP16>(ipt, pv, ju);
  }
}
template <class MT, int VAR, int IPT>
static AnchorFn pick_anchor_pv(bool pv, bool ju) {
  if (!pv) return launch_anchor<MT, false, true, VAR, IPT>;
  if (ju) return launch_anchor<MT, true, true, VAR, IPT>;
  return launch_anchor<MT, true, false, VAR, IPT>;
}
template <class MT, int VAR>
static AnchorFn pick_anchor_ipt(int ipt, bool pv, bool ju) {
  return ipt == 8 ? pick_anchor_pv<MT, VAR, 8>(pv, ju) : pick_anchor_pv<MT, VAR, 4>(pv, ju);
}
template <class MT>
static AnchorFn pick_anchor(int var, int ipt, bool pv, bool ju) {
  switch (var) {
    case VAR_SLICE: return pick_anchor_pv<MT, VAR_SLICE, 4>(pv, ju);
    case VAR_SLICE64: return pick_anchor_pv<MT, VAR_SLICE64, 4>(pv, ju);
    case VAR_SLICEH: return pick_anchor_pv<MT, VAR_SLICEH, 4>(pv, ju);
    case VAR_SLICEB: return pick_anchor_ipt<MT, VAR_SLICEB>(ipt, pv, ju);
    case VAR_WARP: return pick_anchor_ipt<MT, VAR_WARP>(ipt, pv, ju);
    case VAR_WARP4: return pick_anchor_ipt<MT, VAR_WARP4>(ipt, pv, ju);
    default: return pick_anchor_ipt<MT, VAR_WARP16>(ipt, pv, ju);
  }
}
static bool refine_variant(int var) {
  return var == VAR_WARP || var == VAR_WARP4 || var == VAR_WARP16 || var == VAR_WARPL1 ||
         slice_variant(var);
}

static uint32_t tile_items(int var, int ipt) {
  return (uint32_t)((var == VAR_CTA ? SPMV_THREADS : 32) * ipt);
}

// ======================================================================= timing
static thread_local SweepTiming g_timing[3];
static thread_local bool g_timing_on = false;
SweepTiming last_sweep_timing(int phase) {
  return (phase >= 0 && phase < 3) ? g_timing[phase] : SweepTiming{};
}
void set_sweep_timing(bool on) { g_timing_on = on; }

// Algorithmic bytes of one sweep (counted once each): row offsets 4(n+1),
// column indices 4 nnz, values sizeof(MT) nnz, the gathered z once
// (sizeof(VT) n), own y_old and inv_out read, y_new and z_new written
// (4 sizeof(VT) n), plus p when personalised.
static double sweep_bytes(const Operator& op, size_t vt, size_t mt, bool pv) {
  double n = op.n, nnz = (double)op.nnz;
  double b = 4.0 * (n + 1) + 4.0 * nnz + (op.has_vals ? mt * nnz : 0.0) + 5.0 * vt * n;
  if (pv) b += 8.0 * n;
  return b;
}

// Refinement sweep: offsets, indices and FP32 values of the arcs, z_e
// gathered once (4n), y_ref and s_ref read (16n), e and inv_out read (8n),
// e and z_e written (8n), plus p when personalised. The anchor sweep reads
// MT values and the FP64 z once (8n), y_ref (8n) and inv_out (4n), and
// writes s_ref (8n), e and z_e (8n).
static double refine_bytes(const Operator& op, bool pv) {
  double n = op.n, nnz = (double)op.nnz;
  return 4.0 * (n + 1) + 4.0 * nnz + (op.has_vals ? 4.0 * nnz : 0.0) + 36.0 * n +
         (pv ? 8.0 * n : 0.0);
}
static double anchor_bytes(const Operator& op, size_t mt, bool pv) {
  double n = op.n, nnz = (double)op.nnz;
  return 4.0 * (n + 1) + 4.0 * nnz + (op.has_vals ? mt * nnz : 0.0) + 36.0 * n +
         (pv ? 8.0 * n : 0.0);
}

// ======================================================================= phases
struct PhaseResult {
  int32_t iter = 0;
  int32_t converged = 0;
  int32_t stopped = 0;
  double change = 0;
  int launches = 0;
};

// Runs sweeps until the phase's state converges or stops. The host keeps
// one batch of `U` sweeps in flight ahead of the state it inspects, so the
// GPU never waits for the host; sweeps after convergence exit at once.
static PhaseResult run_phase(SweepFn fn, const Operator& op, const Partition& P,
                             const SweepBuffers& B, double d, bool exact, cudaStream_t s,
                             PrWorkspace& ws, IterState* h_state /* pinned, 2 slots */,
                             double* timing_ms, int64_t* timing_n, int32_t iter0 = 0) {
  const int U = 8;
  const unsigned g2 = SPLIT_CTAS;
  PhaseResult r;
  int batch = 0;
  size_t nev = 0;
  bool finished = false;
  auto enqueue = [&](int b) {
    for (int k = 0; k < U; ++k) {
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      if (g_timing_on) {
        e0 = ws.timing_event(nev++);
        e1 = ws.timing_event(nev++);
      }
      fn(op, P, B, k & 1, d, s, g2, e0, e1);
      r.launches += exact ? 3 : 2;
    }
    KNB_CUDA(cudaMemcpyAsync(&h_state[b & 1], B.st, sizeof(IterState), cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaEventRecord(ws.done[b & 1], s));
  };
  enqueue(batch);
  while (!finished) {
    enqueue(batch + 1);
    KNB_CUDA(cudaEventSynchronize(ws.done[batch & 1]));
    const IterState& hs = h_state[batch & 1];
    if (hs.converged || hs.stopped) finished = true;
    ++batch;
  }
  KNB_CUDA(cudaMemcpyAsync(&h_state[0], B.st, sizeof(IterState), cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  const IterState fin = h_state[0];
  if (fin.fault) throw Error("a sweep gave up waiting for its staged arc copies");
  r.iter = fin.iter;
  r.converged = fin.converged;
  r.stopped = fin.stopped;
  r.change = fin.change;
  // Only sweeps that did work count for the timing (later ones exit at once).
  if (g_timing_on) {
    for (size_t k = 0; k + 1 < nev; k += 2) {
      if ((int64_t)(k / 2) < fin.iter - iter0) {
        float ms = 0;
        KNB_CUDA(cudaEventElapsedTime(&ms, ws.pool[k], ws.pool[k + 1]));
        *timing_ms += ms;
        *timing_n += 1;
      }
    }
  }
  return r;
}

static int default_ipt(const Operator& op, int var) {
  (void)op;
  return var == VAR_CTA ? 4 : 8;
}

// ======================================================================= driver
Tuning& tuning() {
  static Tuning t;
  return t;
}

int pagerank_rows(const GraphHandleImpl& g, bool directed) {
  return (g.directed && directed) ? 1 : (g.directed ? 2 : 0);
}

double pagerank_loop_factor(int which, int loops) {
  // Loop factor follows the orientation of the rows (eigenvector.rs:163-169):
  // rows of a directed graph count a loop once unless ignored.
  return loops == 2 ? 0.0 : (which == 1 ? 1.0 : (loops == 0 ? 2.0 : 1.0));
}

void pagerank(GraphHandleImpl& g, const PagerankParams& prm, double* out, bool out_on_device,
              PagerankInfo* info, cudaStream_t s) {
  if (g.n == 0) return;
  const int which = pagerank_rows(g, prm.directed);
  Operator& op = g.op(which, prm.weighted, pagerank_loop_factor(which, prm.loops), s);
  pagerank_op(op, prm, out, out_on_device, info, s);
}

// The operator's PageRank workspace (created on first use).
static PrWorkspace& pr_workspace(Operator& op) {
  std::lock_guard<std::mutex> lock(op.mu);
  if (!op.pr_ws) op.pr_ws = std::make_unique<PrWorkspace>();
  return *static_cast<PrWorkspace*>(op.pr_ws.get());
}

// Pieces of the sliced layout's long rows: a multiple of the resident warps
// at 48 and at 64 warps per SM (192 per SM), so every warp gets as many.
static uint32_t slice_pieces() { return 192u * (uint32_t)device_limits().sms; }

// Milliseconds per sweep of candidate c on operator op: FP32 sweeps (class
// 0, the FP32 phase of mixed solves) or FP64 sweeps (class 1, FP64 solves),
// from the uniform start, the mean of two sweeps after one untimed sweep.
// The state never converges (tolerance -1), so every sweep does its work;
// the solve that follows starts over from its own initial state. Runs
// under the workspace's lock.
static double time_candidate(Operator& op, const SweepPick& c, int cls, bool use32v,
                             PrWorkspace& ws, cudaStream_t s) {
  HotOverride hot(c.hot);
  const bool sl = slice_variant(c.variant);
  const SlicedOp* SO = sl ? &op.sliced((uint32_t)c.long_row, slice_pieces(), s) : nullptr;
  const Relabeled* R = sl ? nullptr : &op.relabeled(s);
  const int ipt = (cls == 0 && !sl) ? 8 : 4;
  static const Partition no_partition;
  const Partition* P = sl ? &no_partition : &op.relabeled_partition(tile_items(c.variant, ipt), s);
  const uint32_t nt = sl ? std::max<uint32_t>(SO->npieces + 1, 64u * (uint32_t)device_limits().sms)
                         : P->ntiles;
  ws.ensure(op.n, nt, cls == 0, cls == 1, false);
  IterState* st = ws.st.get();
  IterState init{};
  init.tol = -1.0;
  init.max_iter = 1 << 30;
  KNB_CUDA(cudaMemcpyAsync(st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
  const unsigned gv = grid_for(op.n, VT_THREADS, 1184);
  SweepFn fn;
  SweepBuffers B{};
  B.v64 = sl ? OpView<double>{} : op.rview64();
  B.v32 = sl ? OpView<float>{} : op.rview32();
  B.part1 = ws.part1.get();
  B.part2 = ws.part2.get();
  B.part3 = ws.part3.get();
  B.st = st;
  B.so = SO;
  if (cls == 0) {
    const float* inv32 = sl ? SO->inv_out32.get() : R->inv_out32.get();
    pr_init<float><<<gv, VT_THREADS, 0, s>>>(ws.y32[0].get(), ws.z32[0].get(), inv32, op.n,
                                              ws.part3.get(), st);
    B.y[0] = ws.y32[0].get(); B.y[1] = ws.y32[1].get();
    B.z[0] = ws.z32[0].get(); B.z[1] = ws.z32[1].get();
    B.inv_out = inv32;
    B.carry = ws.carry32.get();
    B.head = ws.head32.get();
    fn = pick_kernel<float, float, false>(c.variant, ipt, false, true);
  } else {
    const double* inv64 = sl ? SO->inv_out64.get() : R->inv_out64.get();
    pr_init<double><<<gv, VT_THREADS, 0, s>>>(ws.y64[0].get(), ws.z64[0].get(), inv64, op.n,
                                               ws.part3.get(), st);
    B.y[0] = ws.y64[0].get(); B.y[1] = ws.y64[1].get();
    B.z[0] = ws.z64[0].get(); B.z[1] = ws.z64[1].get();
    B.inv_out = inv64;
    B.carry = ws.carry64.get();
    B.head = ws.head64.get();
    fn = use32v ? pick_kernel<double, float, true>(c.variant, ipt, false, true)
                : pick_kernel<double, double, true>(c.variant, ipt, false, true);
  }
  KNB_LAUNCH("pr_init");
  // one untimed sweep, then the fastest of three timed ones (each between its
  // own events), which a passing disturbance of the GPU does not inflate
  constexpr int TIMED = 3;
  fn(op, *P, B, 0, 0.85, s, SPLIT_CTAS, nullptr, nullptr);
  for (int k = 0; k < TIMED; ++k) {
    KNB_CUDA(cudaEventRecord(ws.timing_event(2 * k), s));
    fn(op, *P, B, (k + 1) & 1, 0.85, s, SPLIT_CTAS, nullptr, nullptr);
    KNB_CUDA(cudaEventRecord(ws.timing_event(2 * k + 1), s));
  }
  int32_t fault = 0;
  KNB_CUDA(cudaMemcpyAsync(&fault, &st->fault, sizeof(fault), cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  if (fault) throw Error("a sweep gave up waiting for its staged arc copies");
  double best = 1e300;
  for (int k = 0; k < TIMED; ++k) {
    float ms = 0;
    KNB_CUDA(cudaEventElapsedTime(&ms, ws.timing_event(2 * k), ws.timing_event(2 * k + 1)));
    best = std::min(best, (double)ms);
  }
  return best;
}

// Operators with fewer arcs keep the default sweep: their sweeps take a few
// microseconds, too little to tell the candidates apart.
constexpr uint64_t AUTOTUNE_MIN_ARCS = 1u << 21;

// The sweep kernel for an operator, picked on its first large solve by
// timing each candidate (time_candidate) and kept for the operator's life,
// per precision class (0: solves that start with FP32 sweeps, 1: FP64
// solves). Candidates: the sliced layout at 48 resident warps per SM with
// 24,576, 49,152 or 98,304 FP32 values' worth of L1-allocating columns, at
// 64 warps per SM, with long rows from 64 instead of 255 arcs, and the
// merge-path warp tiles on the layout renumbered by column count; each
// candidate's time is the fastest of three sweeps. Every
// candidate computes the same sums up to rounding; each meets the same
// parity bars (tests/test_gpu_parity.py), and a pinned kernel (net_set_tuning
// keys 4, 7, 10) or key 12 set to 0 bypasses the tuner.
static SweepPick tuned_sweep(Operator& op, int cls, bool use32v, cudaStream_t s) {
  {
    std::lock_guard<std::mutex> lock(op.mu);
    auto it = op.pr_pick.find(cls);
    if (it != op.pr_pick.end()) return it->second;
  }
  PrWorkspace& ws = pr_workspace(op);
  std::lock_guard<std::mutex> ws_lock(ws.mu);
  {
    std::lock_guard<std::mutex> lock(op.mu);  // another thread may have tuned meanwhile
    auto it = op.pr_pick.find(cls);
    if (it != op.pr_pick.end()) return it->second;
  }
  std::vector<SweepPick> cands = {
      {VAR_SLICE, 255, 0, 49152, 0},   {VAR_SLICE, 255, 0, 24576, 0},
      {VAR_SLICE, 255, 0, 98304, 0},   {VAR_SLICE64, 255, 0, 49152, 0},
      {VAR_SLICE, 64, 0, 49152, 0},    {VAR_WARPL1, 0, 0, 24576, 0}};
  // Solves that start with FP32 sweeps run their anchor and refinement
  // sweeps on the FP32 pick, and at 64 warps per SM those are 7-10% slower
  // (R-MAT 24) while its FP32 sweeps are no faster in a solve, though in
  // isolation they can time a few percent ahead: not a candidate there.
  if (cls == 0)
    cands.erase(std::remove_if(cands.begin(), cands.end(),
                               [](const SweepPick& c) { return c.variant == VAR_SLICE64; }),
                cands.end());
  SweepPick best = cands[0];
  best.ms = 1e300;
  for (SweepPick& c : cands) {
    c.ms = time_candidate(op, c, cls, use32v, ws, s);
    if (c.ms < best.ms) best = c;
  }
  // The first candidate stays unless another is clearly faster: two kernels
  // within a few percent of each other trade places from one timing to the
  // next.
  if (best.ms > cands[0].ms * 0.98) best = cands[0];
  std::lock_guard<std::mutex> lock(op.mu);
  op.pr_pick[cls] = best;
  return best;
}

void pagerank_op(Operator& op, const PagerankParams& prm_in, double* out, bool out_on_device,
                 PagerankInfo* info, cudaStream_t s) {
  PagerankParams prm = prm_in;
  const Tuning& tu = tuning();
  if (tu.ipt) prm.ipt = tu.ipt;
  if (tu.variant) prm.variant = tu.variant;
  prm.relabel = prm.relabel && tu.relabel != 0;
  prm.switch_factor = tu.switch_factor;
  prm.switch_floor = tu.switch_floor;
  // the tuned kernel, unless one is pinned (or the operator is small)
  SweepPick pick;
  if (tu.autotune && prm.variant == 0 && prm.ipt == 0 && prm.relabel && tu.long_row == 0 &&
      tu.hot_nodes < 0 && op.nnz >= AUTOTUNE_MIN_ARCS && op.n > 0) {
    const bool use32t = op.has_vals && op.vals32_exact && !prm.fp64_values;
    pick = tuned_sweep(op, prm.precision == PREC_FP64 ? 1 : 0, use32t, s);
    prm.variant = pick.variant;
  }
  HotOverride hot_guard(pick.hot);
  const uint32_t n = op.n;
  if (n == 0) return;
  // Kernel choice (measured on R-MAT scale 24): the sliced layout, 48
  // resident warps per SM, 4 gathers in flight per lane; long rows from 255
  // arcs (the tuner may pick another candidate). Against the merge-path warp
  // tiles on the layout renumbered by column count (kernel 8) it takes the
  // FP32 sweep from 1.20 to 0.85 ms and the FP64 sweep from 1.56 to 0.99 ms.
  // Without renumbering (tuning key 1 set to 0) the merge-path warp tiles
  // run on the operator as built.
  int var32 = prm.variant ? prm.variant : (prm.relabel ? VAR_SLICE : VAR_WARP16);
  int var64 = prm.variant ? prm.variant : (prm.relabel ? VAR_SLICE : VAR_WARP16);
  // The sliced layout numbers nodes its own way, so every phase of a solve
  // on it runs a sliced sweep; the other variants share the renumbering by
  // column count (or none).
  const bool sl = slice_variant(var32) || slice_variant(var64);
  if (sl) {
    if (!slice_variant(var32)) var32 = var64;
    if (!slice_variant(var64)) var64 = var32;
  }
  const bool rl = prm.relabel && !sl;
  // The hot-node sweep needs the renumbered operator: its most gathered
  // nodes come first, and its arc arrays are padded for 16-byte loads.
  if (!rl && (var32 == VAR_HOT || var32 == VAR_HOT16)) var32 = VAR_WARP4;
  if (!rl && (var64 == VAR_HOT || var64 == VAR_HOT16)) var64 = VAR_WARP4;
  int ipt32 = prm.ipt ? prm.ipt : 8;
  int ipt64 = prm.ipt ? prm.ipt : 4;
  // Mixed precision with refinement: one FP64 anchor sweep, then refinement
  // sweeps with FP32 gathers (RefineEpi); both run on warp tiles.
  const bool refine = prm.precision == PREC_MIXED && tu.refine != 0;
  const int var_r =  // refinement
      sl ? var32 : (prm.variant && refine_variant(var32) ? var32 : VAR_WARP16);
  const int ipt_r = (ipt32 == 4 || sl) ? 4 : 8;
  if (refine) {  // the anchor sweep takes the FP64 settings
    if (!refine_variant(var64)) var64 = VAR_WARP16;
    ipt64 = ipt64 == 8 ? 8 : 4;
  }
  // Sliced sweeps keep 4 arcs per lane in flight (8 in FP32 sweeps only when
  // asked for: 0.83 against 0.81 ms on R-MAT 24; wider ones spill).
  if (sl) {
    ipt64 = 4;
    ipt32 = (ipt32 == 8 && prm.ipt == 8 && !slice64_variant(var32)) ? 8 : 4;
  }
  const Relabeled* R = rl ? &op.relabeled(s) : nullptr;
  const SlicedOp* SO =
      sl ? &op.sliced(pick.long_row > 0 ? (uint32_t)pick.long_row
                                        : tu.long_row > 0 ? (uint32_t)tu.long_row : 255u,
                      slice_pieces(), s)
         : nullptr;
  static const Partition no_partition;  // sliced sweeps cut their own work
  const bool mixed_pre = prm.precision == PREC_MIXED || prm.precision == PREC_FP32;
  const Partition* P32 = nullptr;
  const Partition* P64 = nullptr;
  if (mixed_pre) {
    const uint32_t tile = tile_items(var32, ipt32);
    P32 = sl ? &no_partition : rl ? &op.relabeled_partition(tile, s) : &op.partition(tile, s);
  }
  if (prm.precision != PREC_FP32) {
    const uint32_t tile = tile_items(var64, ipt64);
    P64 = sl ? &no_partition : rl ? &op.relabeled_partition(tile, s) : &op.partition(tile, s);
  }
  const Partition* PR = nullptr;
  if (refine) {
    const uint32_t tile = tile_items(var_r, ipt_r);
    PR = sl ? &no_partition : rl ? &op.relabeled_partition(tile, s) : &op.partition(tile, s);
  }
  const OpView<double> v64 = rl ? op.rview64() : op.view64();
  const OpView<float> v32 = rl ? op.rview32() : op.view32();
  const double* inv64 = sl ? SO->inv_out64.get() : rl ? R->inv_out64.get() : op.inv_out64.get();
  const float* inv32 = sl ? SO->inv_out32.get() : rl ? R->inv_out32.get() : op.inv_out32.get();
  const uint32_t* perm = sl ? SO->perm.get() : rl ? R->perm.get() : nullptr;
  const uint32_t* iperm = sl ? SO->iperm.get() : rl ? R->iperm.get() : nullptr;

  const bool pv = prm.personalization != nullptr;
  const bool ju = !pv || prm.dangling == 1;
  const bool mixed = mixed_pre;
  // carries and heads per tile or piece; partials per tile or warp (a
  // sliced sweep leaves one per warp of its grid, at most 64 per SM)
  const uint32_t nt =
      sl ? std::max<uint32_t>(SO->npieces + 1, 64u * (uint32_t)device_limits().sms)
         : std::max({P32 ? P32->ntiles : 0u, P64 ? P64->ntiles : 0u, PR ? PR->ntiles : 0u});
  const unsigned gv = grid_for(n, VT_THREADS, 1184);

  PrWorkspace& ws = pr_workspace(op);
  std::lock_guard<std::mutex> ws_lock(ws.mu);
  ws.ensure(n, nt, mixed, prm.precision != PREC_FP32, pv || !out_on_device);
  IterState* st = ws.st.get();
  IterState* hstate = ws.hstate;

  KNB_CUDA(cudaEventRecord(ws.t0, s));
  if (pv) {
    KNB_CUDA(cudaMemcpyAsync(ws.ptmp.get(), prm.personalization, (size_t)n * 8,
                             prm.pers_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                             s));
    normalize_personalization(ws.ptmp.get(), n, ws.part3.get(), st + 2, hstate + 2, s);
    if (perm) {
      permute_in<<<grid_for(n, 256), 256, 0, s>>>(ws.ptmp.get(), perm, n, ws.pvec.get());
      KNB_LAUNCH("permute_in");
    } else {
      KNB_CUDA(cudaMemcpyAsync(ws.pvec.get(), ws.ptmp.get(), (size_t)n * 8,
                               cudaMemcpyDeviceToDevice, s));
    }
  }
  const double* pdev = pv ? ws.pvec.get() : nullptr;

  IterState init{};
  int launches = pv ? 3 : 0;
  double tms32 = 0, tms64 = 0, tmsr = 0;
  int64_t tn32 = 0, tn64 = 0, tnr = 0;
  PhaseResult r32, r64;
  const int64_t cap = prm.max_iter;
  double tol32 = std::max(prm.tol * prm.switch_factor, prm.switch_floor);
  if (prm.precision == PREC_FP32) tol32 = prm.tol;

  if (mixed) {
    init.tol = tol32;
    init.max_iter = (int32_t)std::min<int64_t>(cap, INT32_MAX);
    KNB_CUDA(cudaMemcpyAsync(st, &init, sizeof(init), cudaMemcpyHostToDevice, s));
    pr_init<float><<<gv, VT_THREADS, 0, s>>>(ws.y32[0].get(), ws.z32[0].get(), inv32, n,
                                              ws.part3.get(), st);
    KNB_LAUNCH("pr_init");
    ++launches;
    SweepBuffers B{v64, v32, {ws.y32[0].get(), ws.y32[1].get()},
                   {ws.z32[0].get(), ws.z32[1].get()}, inv32, pdev, ws.carry32.get(),
                   ws.head32.get(), ws.part1.get(), ws.part2.get(), ws.part3.get(), st};
    B.so = SO;
    SweepFn fn = pick_kernel<float, float, false>(var32, ipt32, pv, ju);
    r32 = run_phase(fn, op, *P32, B, prm.damping, false, s, ws, hstate, &tms32, &tn32);
    launches += r32.launches;
    if (r32.stopped && !r32.converged)
      throw Error("PageRank did not converge to tolerance " + std::to_string(prm.tol) +
                  " within " + std::to_string(prm.max_iter) + " iterations");
  }
  const float* y32_last = mixed ? ws.y32[r32.iter & 1].get() : nullptr;
  if (prm.precision != PREC_FP32) {
    IterState i64{};
    i64.tol = prm.tol;
    i64.max_iter = (int32_t)std::min<int64_t>(cap - r32.iter, INT32_MAX);
    if (i64.max_iter <= 0) i64.max_iter = 1;
    KNB_CUDA(cudaMemcpyAsync(st + 1, &i64, sizeof(i64), cudaMemcpyHostToDevice, s));
    if (mixed) {
      pr_switch<<<gv, VT_THREADS, 0, s>>>(y32_last, st, ws.y64[0].get(), ws.z64[0].get(), inv64,
                                          n, ws.part3.get(), st + 1);
      KNB_LAUNCH("pr_switch");
    } else {
      pr_init<double><<<gv, VT_THREADS, 0, s>>>(ws.y64[0].get(), ws.z64[0].get(), inv64, n,
                                                 ws.part3.get(), st + 1);
      KNB_LAUNCH("pr_init");
    }
    ++launches;
    bool use32 = op.has_vals && op.vals32_exact && !prm.fp64_values;
    if (refine) {
      // y_ref = y64[0] (from pr_switch), s_ref in z64[1]; e and z_e reuse
      // the FP32 iterate buffers, free once pr_switch has read them.
      SweepBuffers R{v64, v32, {ws.y32[0].get(), ws.y32[1].get()},
                     {ws.z32[0].get(), ws.z32[1].get()}, inv32, pdev, ws.carry32.get(),
                     ws.head32.get(), ws.part1.get(), ws.part2.get(), ws.part3.get(), st + 1,
                     ws.y64[0].get(), ws.z64[1].get(), SO};
      AnchorFn af = use32 ? pick_anchor<float>(var64, ipt64, pv, ju)
                          : pick_anchor<double>(var64, ipt64, pv, ju);
      af(op, *P64, R, ws.z64[0].get(), ws.carry64.get(), ws.head64.get(), prm.damping, s,
         SPLIT_CTAS, g_timing_on ? ws.a0 : nullptr, g_timing_on ? ws.a1 : nullptr);
      launches += 3;
      SweepFn fr = pick_refine(var_r, ipt_r, pv, ju);
      r64 = run_phase(fr, op, *PR, R, prm.damping, true, s, ws, hstate, &tmsr, &tnr, 1);
      if (g_timing_on) {
        float ms = 0;
        KNB_CUDA(cudaEventElapsedTime(&ms, ws.a0, ws.a1));
        tms64 += ms;
        tn64 += 1;
      }
    } else {
      SweepBuffers B{v64, v32, {ws.y64[0].get(), ws.y64[1].get()},
                     {ws.z64[0].get(), ws.z64[1].get()}, inv64, pdev, ws.carry64.get(),
                     ws.head64.get(), ws.part1.get(), ws.part2.get(), ws.part3.get(), st + 1};
      B.so = SO;
      SweepFn fn = use32 ? pick_kernel<double, float, true>(var64, ipt64, pv, ju)
                         : pick_kernel<double, double, true>(var64, ipt64, pv, ju);
      r64 = run_phase(fn, op, *P64, B, prm.damping, true, s, ws, hstate, &tms64, &tn64);
    }
    launches += r64.launches;
    if (!r64.converged)
      throw Error("PageRank did not converge to tolerance " + std::to_string(prm.tol) +
                  " within " + std::to_string(prm.max_iter) + " iterations");
  }
  // output, in the caller's node order
  double* outp = out_on_device ? out : ws.dout.get();
  if (!out_on_device && !outp) {
    ws.dout.alloc(n);
    outp = ws.dout.get();
  }
  if (prm.precision == PREC_FP32) {
    pr_output<float><<<gv, VT_THREADS, 0, s>>>(y32_last, st, n, iperm, outp);
  } else if (refine) {
    pr_output_ref<<<gv, VT_THREADS, 0, s>>>(ws.y64[0].get(), ws.y32[(r64.iter - 1) & 1].get(),
                                            st + 1, n, iperm, outp);
  } else {
    pr_output<double><<<gv, VT_THREADS, 0, s>>>(ws.y64[r64.iter & 1].get(), st + 1, n, iperm,
                                                 outp);
  }
  KNB_LAUNCH("pr_output");
  ++launches;
  if (!out_on_device)
    KNB_CUDA(cudaMemcpyAsync(out, outp, (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaEventRecord(ws.t1, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  KNB_CUDA(cudaEventElapsedTime(&ms, ws.t0, ws.t1));
  if (info) {
    info->iterations = r32.iter + r64.iter;
    info->iterations_fp32 = r32.iter;
    info->change = prm.precision == PREC_FP32 ? r32.change : r64.change;
    info->seconds = ms * 1e-3;
    info->converged = 1;
    info->kernel_launches = launches;
    info->sweep_kernel = prm.precision == PREC_FP64 ? var64 : var32;
    info->long_row = sl ? (int32_t)SO->lw : 0;
    info->hot_columns = (int32_t)(hot_setting() >= 0 ? hot_setting() : sl ? 49152 : 24576);
  }
  const bool use32v = op.has_vals && op.vals32_exact && !prm.fp64_values;
  g_timing[0] = {tn32, tms32, sweep_bytes(op, 4, 4, pv)};
  g_timing[1] = {tn64, tms64,
                 refine ? anchor_bytes(op, use32v ? 4 : 8, pv)
                        : sweep_bytes(op, 8, use32v ? 4 : 8, pv)};
  g_timing[2] = {tnr, tmsr, refine_bytes(op, pv)};
}

}  // namespace knb
