// Batched personalised PageRank: B teleport vectors solved together as a
// sparse matrix times dense matrix iteration (SpMM). Each column is the
// reference's PageRank with that personalization vector
// (crates/engine/src/metrics/spectral.rs:211-281): it has its own
// normalisation, dangling mass and L1 change, and it stops at its own first
// sweep with change <= tol, keeping that iterate while the others go on.
//
// Layout: the iterate is node-major, Y[i * B + c], so the gather of a source
// node's B values is one contiguous run (coalesced across the warp: lane l
// holds columns l, l + 32, ...). Rows are split over warps in ranges of
// about equal arc counts; rows with more than LONG_ROW arcs are cut into
// chunks whose partial sums a second kernel adds in chunk order. Per-column
// sums are kept per lane, joined per CTA in warp order and per sweep in CTA
// order, so the results do not change from run to run.
//
// Precision: FP64, or mixed (FP32 sweeps until every column's change is below
// max(tol * switch_factor, switch_floor), then, on the same trajectories, one
// FP64 anchor sweep and refinement sweeps gathering the FP32 correction (or
// plain FP64 sweeps) until each column meets tol).
#include <algorithm>
#include <cfloat>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <vector>

#include "batch.cuh"
#include "pagerank.cuh"

namespace knb {

constexpr int BT = 256;          // threads per CTA
constexpr int BW = BT / 32;      // warps per CTA
constexpr int MAXVW = 8;         // columns per lane (B <= 256 per launch)
constexpr uint32_t LONG_ROW = 512;
constexpr uint32_t RANGE_ARCS = 256;

struct RowRange {
  uint32_t lo, hi;
};
struct Chunk {
  uint32_t row, a0, a1;
};

// Per-column state of a batch phase.
struct ColState {
  double inv_total;       // 1 / sum of the column's current iterate
  double dterm;           // its dangling mass, normalised
  double prev_inv_total;
  double total, change;
  int32_t frozen;         // converged (or finished) columns keep their iterate
  int32_t iter;           // sweeps this column took
  int32_t converged;
  int32_t pad;
};

struct BatchScalars {
  double d;
  double pu;    // 1 / n
  uint32_t n, B;
  int jump_uniform;
  double tol;
  int32_t max_iter;
  int32_t exact;
};

// Arcs whose gathers one warp keeps in flight together (U): 1, 2 or 4,
// picked per operator by timing (tune_arcs_in_flight). The products are
// added in arc order whatever U is, so the choice never changes a result.
constexpr int U_CANDIDATES[] = {1, 2, 4};

// The normalised teleport columns: dense node-major P[i * B + c], or, when
// few entries are nonzero, each row's nonzero (column, value) pairs in
// column order (rowptr over n + 1 rows).
struct PersView {
  const double* dense;
  const uint32_t* rowptr;
  const uint32_t* cols;
  const double* vals;
};

// Row sum of one row of A times Z for this lane's columns. U arcs at a
// time: their indices, then all their gathers, then the products added in
// arc order (so each column's sum keeps the order of a one-arc loop).
template <class VT, class MT, int VW, int U>
__device__ __forceinline__ void row_product(const OpView<MT>& op, const VT* __restrict__ Z,
                                            uint32_t B, uint32_t a0, uint32_t a1, int lane,
                                            VT (&acc)[VW]) {
#pragma unroll
  for (int v = 0; v < VW; ++v) acc[v] = VT(0);
  uint32_t k = a0;
  for (; k + U <= a1; k += U) {
    uint32_t j[U];
    VT w[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      j[u] = __ldg(op.cols + k + u);
      w[u] = op.vals ? (VT)__ldg(op.vals + k + u) : VT(1);
    }
    VT z[U][VW];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const VT* zr = Z + (size_t)j[u] * B;
#pragma unroll
      for (int v = 0; v < VW; ++v) {
        const uint32_t c = lane + 32 * v;
        z[u][v] = c < B ? __ldg(zr + c) : VT(0);
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u)
#pragma unroll
      for (int v = 0; v < VW; ++v)
        if (lane + 32 * v < B) acc[v] += w[u] * z[u][v];
  }
  for (; k < a1; ++k) {
    const uint32_t j = __ldg(op.cols + k);
    const VT w = op.vals ? (VT)__ldg(op.vals + k) : VT(1);
    const VT* zr = Z + (size_t)j * B;
#pragma unroll
    for (int v = 0; v < VW; ++v) {
      const uint32_t c = lane + 32 * v;
      if (c < B) acc[v] += w * __ldg(zr + c);
    }
  }
}

// Epilogue modes: the plain update (VT iterate), the anchor sweep and the
// refinement sweeps of the mixed path's FP64 phase. As in the single-vector
// path (RefineEpi, pagerank.cu) each column's iterate is held from the
// anchor on as y = y_ref + e with e in FP32: the anchor sweep gathers the
// FP64 z_ref = y_ref / out and keeps s_ref = A z_ref; a refinement sweep
// gathers z_e = e / out in FP32 and forms s = s_ref + A z_e, the update, the
// sums and the change in FP64. A refinement sweep gathers B FP32 values per
// arc where an FP64 sweep gathers B FP64 values.
enum { EPI_PLAIN = 0, EPI_ANCHOR = 1, EPI_REFINE = 2 };
struct RefineBufs {
  const double* yref;  // n x B: the iterate the anchor sweep starts from
  double* sref;        // n x B: A z_ref, written by the anchor sweep
  const float* eold;   // refinement sweeps: e of the input iterate
  float* enew;         // e of the new iterate
  float* zenew;        // enew / out
  const float* io32;   // 1 / out in FP32 (0 for dangling nodes)
};

// The PageRank update of row i for this lane's columns, and its per-column
// sums (mass, dangling mass, L1 change) into the warp's slice red[3][B] of
// shared memory (column c belongs to lane c mod 32, so every slot has one
// writer and takes its rows in order).
template <class VT, int VW, int MODE>
__device__ __forceinline__ void row_update(uint32_t i, const VT (&s)[VW], int lane,
                                           const BatchScalars& bs, const ColState* cs,
                                           const VT* __restrict__ Yold, VT* __restrict__ Ynew,
                                           VT* __restrict__ Znew, const VT* __restrict__ inv_out,
                                           const PersView& pv, const RefineBufs& rb,
                                           double* red) {
  using PT = std::conditional_t<MODE == EPI_PLAIN, VT, double>;
  PT psp[VW];  // this lane's teleport values of row i (sparse teleport)
#pragma unroll
  for (int v = 0; v < VW; ++v) psp[v] = PT(0);
  if (!pv.dense) {
    for (uint32_t e = pv.rowptr[i]; e < pv.rowptr[i + 1]; ++e) {
      const uint32_t c = pv.cols[e];
      if ((c & 31u) != (uint32_t)lane) continue;
      const PT x = (PT)pv.vals[e];
#pragma unroll
      for (int v = 0; v < VW; ++v)
        if ((c >> 5) == (uint32_t)v) psp[v] = x;
    }
  }
  if constexpr (MODE == EPI_PLAIN) {
    const VT io = inv_out[i];
#pragma unroll
    for (int v = 0; v < VW; ++v) {
      const uint32_t c = lane + 32 * v;
      if (c >= bs.B || cs[c].frozen) continue;
      const VT it = (VT)cs[c].inv_total, dt = (VT)cs[c].dterm;
      const size_t q = (size_t)i * bs.B + c;
      const VT pg = pv.dense ? (VT)pv.dense[q] : psp[v];
      const VT jg = bs.jump_uniform ? (VT)bs.pu : pg;
      const VT u = (VT)bs.d * (s[v] * it + dt * jg) + (VT)(1.0 - bs.d) * pg;
      const VT xo = Yold[q] * it;
      Ynew[q] = u;
      Znew[q] = u * io;
      red[c] += (double)u;
      if (io == VT(0)) red[bs.B + c] += (double)u;
      red[2 * bs.B + c] += fabs((double)u - (double)xo);
    }
  } else {
    (void)Yold;
    (void)Ynew;
    (void)Znew;
    (void)inv_out;
    const float io = rb.io32[i];
#pragma unroll
    for (int v = 0; v < VW; ++v) {
      const uint32_t c = lane + 32 * v;
      if (c >= bs.B || cs[c].frozen) continue;
      const double it = cs[c].inv_total, dt = cs[c].dterm;
      const size_t q = (size_t)i * bs.B + c;
      double sum;
      if constexpr (MODE == EPI_ANCHOR) {
        sum = (double)s[v];
        rb.sref[q] = sum;
      } else {
        sum = rb.sref[q] + (double)s[v];
      }
      const double pg = pv.dense ? pv.dense[q] : psp[v];
      const double jg = bs.jump_uniform ? bs.pu : pg;
      const double u = bs.d * (sum * it + dt * jg) + (1.0 - bs.d) * pg;
      const double yr = rb.yref[q];
      const double yo = MODE == EPI_ANCHOR ? yr : yr + (double)rb.eold[q];
      const float en = (float)(u - yr);
      const double us = yr + (double)en;  // the iterate as stored
      rb.enew[q] = en;
      rb.zenew[q] = en * io;
      red[c] += us;
      if (io == 0.0f) red[bs.B + c] += us;
      red[2 * bs.B + c] += fabs(us - yo * it);
    }
  }
}

// Zeroes this warp's slice [3][B] of the per-warp column sums in smem.
__device__ __forceinline__ double* warp_sums(double* smem, uint32_t B) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double* red = smem + (size_t)w * 3 * B;
  for (uint32_t q = lane; q < 3 * B; q += 32) red[q] = 0.0;
  __syncwarp();
  return red;
}

// Joins the warps' per-column sums of a CTA (smem [BW][3][B]) in warp order
// into part[cta][3][B].
__device__ __forceinline__ void cta_column_sums(uint32_t B, double* __restrict__ part,
                                                const double* smem) {
  __syncthreads();
  for (uint32_t q = threadIdx.x; q < 3 * B; q += BT) {
    double a = 0;
    for (int ww = 0; ww < BW; ++ww) a += smem[(size_t)ww * 3 * B + q];
    part[(size_t)blockIdx.x * 3 * B + q] = a;
  }
}

template <class VT, class MT, int VW, int U, int MODE>
__global__ void __launch_bounds__(BT)
spmm_rows(OpView<MT> op, const VT* __restrict__ Z, const RowRange* __restrict__ ranges,
          uint32_t nranges, BatchScalars bs, const ColState* __restrict__ cs,
          const VT* __restrict__ Yold, VT* __restrict__ Ynew, VT* __restrict__ Znew,
          const VT* __restrict__ inv_out, PersView P, RefineBufs rb,
          double* __restrict__ part, const int32_t* __restrict__ all_frozen) {
  if (*all_frozen) return;
  extern __shared__ double smem_b[];
  const int lane = threadIdx.x & 31;
  double* red = warp_sums(smem_b, bs.B);
  const uint32_t gw = blockIdx.x * BW + (threadIdx.x >> 5), nw = gridDim.x * BW;
  for (uint32_t r = gw; r < nranges; r += nw) {
    const RowRange rr = ranges[r];
    for (uint32_t i = rr.lo; i < rr.hi; ++i) {
      const uint32_t a0 = op.off[i], a1 = op.off[i + 1];
      if (a1 - a0 > LONG_ROW) continue;  // long rows: spmm_chunks / spmm_long
      VT acc[VW];
      row_product<VT, MT, VW, U>(op, Z, bs.B, a0, a1, lane, acc);
      row_update<VT, VW, MODE>(i, acc, lane, bs, cs, Yold, Ynew, Znew, inv_out, P, rb, red);
    }
  }
  cta_column_sums(bs.B, part, smem_b);
}

// Partial products of the chunks of long rows.
template <class VT, class MT, int VW, int U>
__global__ void __launch_bounds__(BT)
spmm_chunks(OpView<MT> op, const VT* __restrict__ Z, const Chunk* __restrict__ chunks,
            uint32_t nchunks, uint32_t B, VT* __restrict__ scratch,
            const int32_t* __restrict__ all_frozen) {
  if (*all_frozen) return;
  const int lane = threadIdx.x & 31;
  const uint32_t gw = blockIdx.x * BW + (threadIdx.x >> 5), nw = gridDim.x * BW;
  for (uint32_t q = gw; q < nchunks; q += nw) {
    const Chunk ch = chunks[q];
    VT acc[VW];
    row_product<VT, MT, VW, U>(op, Z, B, ch.a0, ch.a1, lane, acc);
#pragma unroll
    for (int v = 0; v < VW; ++v) {
      const uint32_t c = lane + 32 * v;
      if (c < B) scratch[(size_t)q * B + c] = acc[v];
    }
  }
}

// Long rows: chunk partials added in chunk order, then the update.
template <class VT, int VW, int MODE>
__global__ void __launch_bounds__(BT)
spmm_long(const uint32_t* __restrict__ lrow, const uint32_t* __restrict__ lfirst, uint32_t nlong,
          const VT* __restrict__ scratch, BatchScalars bs, const ColState* __restrict__ cs,
          const VT* __restrict__ Yold, VT* __restrict__ Ynew, VT* __restrict__ Znew,
          const VT* __restrict__ inv_out, PersView P, RefineBufs rb,
          double* __restrict__ part, const int32_t* __restrict__ all_frozen) {
  if (*all_frozen) return;
  extern __shared__ double smem_b[];
  const int lane = threadIdx.x & 31;
  double* red = warp_sums(smem_b, bs.B);
  const uint32_t gw = blockIdx.x * BW + (threadIdx.x >> 5), nw = gridDim.x * BW;
  for (uint32_t q = gw; q < nlong; q += nw) {
    VT acc[VW];
#pragma unroll
    for (int v = 0; v < VW; ++v) acc[v] = VT(0);
    for (uint32_t k = lfirst[q]; k < lfirst[q + 1]; ++k)
#pragma unroll
      for (int v = 0; v < VW; ++v) {
        const uint32_t c = lane + 32 * v;
        if (c < bs.B) acc[v] += scratch[(size_t)k * bs.B + c];
      }
    row_update<VT, VW, MODE>(lrow[q], acc, lane, bs, cs, Yold, Ynew, Znew, inv_out, P, rb, red);
  }
  cta_column_sums(bs.B, part, smem_b);
}

// Per column: sums over the CTAs in order, the stopping rule, the scalars of
// the next sweep; then whether every column is frozen.
__global__ void spmm_finish(const double* __restrict__ part, uint32_t nparts, BatchScalars bs,
                            ColState* cs, int32_t* all_frozen, int32_t count_sweep) {
  __shared__ int any_active;
  if (threadIdx.x == 0) any_active = 0;
  __syncthreads();
  if (*all_frozen) return;
  for (uint32_t c = threadIdx.x; c < bs.B; c += blockDim.x) {
    ColState s = cs[c];
    if (!s.frozen) {
      double T = 0, D = 0, ch = 0;
      for (uint32_t q = 0; q < nparts; ++q) {
        const double* p = part + (size_t)q * 3 * bs.B;
        T += p[c];
        D += p[bs.B + c];
        ch += p[2 * bs.B + c];
      }
      s.prev_inv_total = s.inv_total;
      s.total = T;
      s.inv_total = 1.0 / T;
      s.dterm = D / T;
      s.change = ch;
      s.iter += count_sweep;
      if (ch <= bs.tol) {
        s.converged = 1;
        s.frozen = 1;
      } else if (s.iter >= bs.max_iter) {
        s.frozen = 1;
      }
      cs[c] = s;
    }
    if (!s.frozen) atomicOr(&any_active, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0 && !any_active) *all_frozen = 1;
}

// Start: Y = 1/n, Z = Y / out, per-column dangling mass (fixed-order sums).
template <class VT>
__global__ void spmm_init(VT* __restrict__ Y, VT* __restrict__ Zb, const VT* __restrict__ inv_out,
                          uint32_t n, uint32_t B, double* __restrict__ colD) {
  // one CTA per column group of 256 threads: thread c sums column c's dangling mass
  const VT x0 = (VT)(1.0 / (double)n);
  const uint64_t total = (uint64_t)n * B;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(q / B);
    Y[q] = x0;
    Zb[q] = x0 * inv_out[i];
  }
  (void)colD;
}

// Dangling count (same for every column at the start): D0 = n_dangling / n.
__global__ void spmm_set_state(ColState* cs, uint32_t B, double dterm0, int32_t max_iter) {
  for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < B; c += gridDim.x * blockDim.x) {
    ColState s{};
    s.inv_total = 1.0;
    s.prev_inv_total = 1.0;
    s.dterm = dterm0;
    s.total = 1.0;
    cs[c] = s;
  }
  (void)max_iter;
}

// FP32 -> FP64 hand-over: Y64 = Y32 / T per column, read from the buffer the
// column's FP32 phase stopped in; Z64 = Y64 / out.
__global__ void spmm_switch(const float* __restrict__ Y0, const float* __restrict__ Y1,
                            const ColState* __restrict__ cs32, double* __restrict__ Y64,
                            double* __restrict__ Z64, const double* __restrict__ inv_out,
                            uint32_t n, uint32_t B) {
  const uint64_t total = (uint64_t)n * B;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(q / B), c = (uint32_t)(q % B);
    const ColState s = cs32[c];
    const float* Y = (s.iter & 1) ? Y1 : Y0;
    const double y = (double)Y[q] * s.inv_total;
    Y64[q] = y;
    Z64[q] = y * inv_out[i];
  }
}

// Column sums (and dangling sums) of a node-major n x B matrix: CTA b adds
// rows b, b + G, ... per column (thread c owns column c), then one CTA adds
// the CTA partials in order and writes the column states.
__global__ void column_sums_part(const double* __restrict__ Y, const double* __restrict__ inv_out,
                                 uint32_t n, uint32_t B, double* __restrict__ part) {
  const uint32_t c = threadIdx.x;
  if (c >= B) return;
  double T = 0, D = 0;
  for (uint32_t i = blockIdx.x; i < n; i += gridDim.x) {
    const double y = Y[(size_t)i * B + c];
    T += y;
    if (inv_out[i] == 0.0) D += y;
  }
  part[(size_t)blockIdx.x * 2 * B + c] = T;
  part[(size_t)blockIdx.x * 2 * B + B + c] = D;
}

__global__ void column_sums_finish(const double* __restrict__ part, uint32_t nparts, uint32_t B,
                                   ColState* cs) {
  const uint32_t c = threadIdx.x;
  if (c >= B) return;
  double T = 0, D = 0;
  for (uint32_t q = 0; q < nparts; ++q) {
    T += part[(size_t)q * 2 * B + c];
    D += part[(size_t)q * 2 * B + B + c];
  }
  ColState s{};
  s.total = T;
  s.inv_total = 1.0 / T;
  s.prev_inv_total = s.inv_total;
  s.dterm = D / T;
  cs[c] = s;
}

// Personalization: column-major input (p[c * n + i]) checked and rescaled per
// column, stored node-major.
__global__ void pers_columns(const double* __restrict__ pin, uint32_t n, uint32_t B,
                             double* __restrict__ pnm, int32_t* __restrict__ bad,
                             double* __restrict__ sums) {
  // one warp per column: fixed-order sum
  const int lane = threadIdx.x & 31;
  for (uint32_t c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); c < B;
       c += gridDim.x * (blockDim.x / 32)) {
    double a = 0;
    int b = 0;
    for (uint32_t i = lane; i < n; i += 32) {
      double v = pin[(size_t)c * n + i];
      if (!isfinite(v) || v < 0.0) b = 1;
      else a += v;
    }
    a = warp_sum(a);
    b = __any_sync(0xffffffffu, b);
    if (lane == 0) {
      sums[c] = a;
      if (b || !(a > 0.0)) atomicOr(bad, b ? 1 : 2);
    }
  }
}

__global__ void pers_scatter(const double* __restrict__ pin, const double* __restrict__ sums,
                             uint32_t n, uint32_t B, double* __restrict__ pnm) {
  const uint64_t total = (uint64_t)n * B;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(q / B), c = (uint32_t)(q % B);
    pnm[q] = pin[(size_t)c * n + i] / sums[c];
  }
}

// Nonzero teleport entries per node of a column group (column-major input).
__global__ void pers_row_counts(const double* __restrict__ pin, uint32_t n, uint32_t B,
                                uint32_t* __restrict__ cnt) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t k = 0;
    for (uint32_t c = 0; c < B; ++c) k += pin[(size_t)c * n + i] != 0.0 ? 1u : 0u;
    cnt[i] = k;
  }
}

// Each node's nonzero entries, normalised as pers_scatter does, in column order.
__global__ void pers_row_fill(const double* __restrict__ pin, const double* __restrict__ sums,
                              uint32_t n, uint32_t B, const uint32_t* __restrict__ rowptr,
                              uint32_t* __restrict__ cols, double* __restrict__ vals) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t e = rowptr[i];
    for (uint32_t c = 0; c < B; ++c) {
      const double v = pin[(size_t)c * n + i];
      if (v != 0.0) {
        cols[e] = c;
        vals[e] = v / sums[c];
        ++e;
      }
    }
  }
}

// Output: column-major out[c * n + i] = Y_c[i] / T_c from the buffer the
// column stopped in.
template <class VT>
__global__ void spmm_output(const VT* __restrict__ Y0, const VT* __restrict__ Y1,
                            const ColState* __restrict__ cs, uint32_t n, uint32_t B,
                            double* __restrict__ out) {
  const uint64_t total = (uint64_t)n * B;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(q % n), c = (uint32_t)(q / n);
    const ColState s = cs[c];
    const VT* Y = (s.iter & 1) ? Y1 : Y0;
    out[q] = (double)Y[(size_t)i * B + c] / s.total;
  }
}

// Output of a refined phase: (y_ref + e) / total per column, e read from the
// buffer of the column's last sweep.
__global__ void spmm_output_ref(const double* __restrict__ Yref, const float* __restrict__ E0,
                                const float* __restrict__ E1, const ColState* __restrict__ cs,
                                uint32_t n, uint32_t B, double* __restrict__ out) {
  const uint64_t total = (uint64_t)n * B;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < total;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(q % n), c = (uint32_t)(q / n);
    const ColState s = cs[c];
    const float* E = (s.iter & 1) ? E1 : E0;
    const size_t r = (size_t)i * B + c;
    out[q] = (Yref[r] + (double)E[r]) / s.total;
  }
}

// ----------------------------------------------------------------------- host
struct BatchPlan {
  std::vector<RowRange> ranges;
  std::vector<Chunk> chunks;
  std::vector<uint32_t> lrow, lfirst;
};

static BatchPlan make_plan(const std::vector<uint32_t>& off, uint32_t n) {
  BatchPlan p;
  uint32_t lo = 0;
  uint64_t acc = 0;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t deg = off[i + 1] - off[i];
    if (deg > LONG_ROW) {
      p.lrow.push_back(i);
      p.lfirst.push_back((uint32_t)p.chunks.size());
      for (uint32_t a = off[i]; a < off[i + 1]; a += LONG_ROW)
        p.chunks.push_back({i, a, std::min(off[i + 1], a + LONG_ROW)});
    } else {
      acc += deg + 1;
    }
    if (acc >= RANGE_ARCS) {
      p.ranges.push_back({lo, i + 1});
      lo = i + 1;
      acc = 0;
    }
  }
  if (lo < n) p.ranges.push_back({lo, n});
  p.lfirst.push_back((uint32_t)p.chunks.size());
  return p;
}

template <class T>
static void upload(DevBuf<T>& d, const std::vector<T>& h, cudaStream_t s) {
  d.alloc(std::max<size_t>(h.size(), 1));
  if (!h.empty()) KNB_CUDA(cudaMemcpyAsync(d.get(), h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
}

// One sweep: the row products and updates, then (finish) the per-column
// sums, stopping rule and next sweep's scalars. Without finish the sweep
// only rewrites Ynew, Znew, the chunk scratch and the partials.
template <class VT, class MT, int VW, int U, int MODE>
static int batch_sweep(const OpView<MT>& op, const DevBuf<RowRange>& ranges, uint32_t nranges,
                       const DevBuf<Chunk>& chunks, uint32_t nchunks, const DevBuf<uint32_t>& lrow,
                       const DevBuf<uint32_t>& lfirst, uint32_t nlong, const BatchScalars& bs,
                       ColState* cs, const VT* Yold, VT* Ynew, const VT* Zold, VT* Znew,
                       const VT* inv_out, const PersView& P, const RefineBufs& rb, VT* scratch,
                       double* part, int32_t* all_frozen, unsigned grid, bool finish,
                       cudaStream_t s) {
  const size_t smem = (size_t)BW * 3 * bs.B * sizeof(double);
  set_func_attr((const void*)spmm_rows<VT, MT, VW, U, MODE>,
                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(BW * 3 * 256 * sizeof(double)));
  set_func_attr((const void*)spmm_long<VT, VW, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                (int)(BW * 3 * 256 * sizeof(double)));
  int launches = 0;
  if (nchunks) {
    spmm_chunks<VT, MT, VW, U><<<grid, BT, 0, s>>>(op, Zold, chunks.get(), nchunks, bs.B, scratch,
                                                    all_frozen);
    ++launches;
  }
  spmm_rows<VT, MT, VW, U, MODE><<<grid, BT, smem, s>>>(op, Zold, ranges.get(), nranges, bs, cs,
                                                        Yold, Ynew, Znew, inv_out, P, rb, part,
                                                        all_frozen);
  spmm_long<VT, VW, MODE><<<grid, BT, smem, s>>>(lrow.get(), lfirst.get(), nlong, scratch, bs, cs,
                                                 Yold, Ynew, Znew, inv_out, P, rb,
                                                 part + (size_t)grid * 3 * bs.B, all_frozen);
  if (finish) spmm_finish<<<1, 256, 0, s>>>(part, 2 * grid, bs, cs, all_frozen, 1);
  KNB_LAUNCH("batch sweep");
  return launches + (finish ? 3 : 2);
}

template <class VT, class MT, int MODE = EPI_PLAIN>
static int batch_sweep_vw(int vw, int u, const OpView<MT>& op, const DevBuf<RowRange>& ranges,
                          uint32_t nranges, const DevBuf<Chunk>& chunks, uint32_t nchunks,
                          const DevBuf<uint32_t>& lrow, const DevBuf<uint32_t>& lfirst,
                          uint32_t nlong, const BatchScalars& bs, ColState* cs, const VT* Yold,
                          VT* Ynew, const VT* Zold, VT* Znew, const VT* inv_out, const PersView& P,
                          VT* scratch, double* part, int32_t* all_frozen, unsigned grid,
                          cudaStream_t s, bool finish = true, const RefineBufs& rb = RefineBufs{}) {
#define KNB_SW(V, UU)                                                                             \
  return batch_sweep<VT, MT, V, UU, MODE>(op, ranges, nranges, chunks, nchunks, lrow, lfirst,     \
                                          nlong, bs, cs, Yold, Ynew, Zold, Znew, inv_out, P, rb,  \
                                          scratch, part, all_frozen, grid, finish, s)
#define KNB_SWU(V)                   \
  switch (u) {                       \
    case 1: KNB_SW(V, 1);            \
    case 2: KNB_SW(V, 2);            \
    default: KNB_SW(V, 4);           \
  }
  switch (vw) {
    case 1: KNB_SWU(1);
    case 2: KNB_SWU(2);
    case 4: KNB_SWU(4);
    default: KNB_SWU(8);
  }
#undef KNB_SWU
#undef KNB_SW
}

// Times one sweep of each arcs-in-flight candidate on the phase's starting
// state (without the finish, so nothing but buffers the first real sweep
// rewrites is touched) and returns the fastest.
template <class VT, class MT>
static int tune_arcs_in_flight(int vw, const OpView<MT>& op, const DevBuf<RowRange>& ranges,
                               uint32_t nranges, const DevBuf<Chunk>& chunks, uint32_t nchunks,
                               const DevBuf<uint32_t>& lrow, const DevBuf<uint32_t>& lfirst,
                               uint32_t nlong, const BatchScalars& bs, ColState* cs,
                               const VT* Yold, VT* Ynew, const VT* Zold, VT* Znew,
                               const VT* inv_out, const PersView& P, VT* scratch, double* part,
                               int32_t* all_frozen, unsigned grid, cudaStream_t s) {
  cudaEvent_t e0, e1;
  KNB_CUDA(cudaEventCreate(&e0));
  KNB_CUDA(cudaEventCreate(&e1));
  int best = U_CANDIDATES[0];
  float best_ms = 0;
  for (int u : U_CANDIDATES) {
    KNB_CUDA(cudaEventRecord(e0, s));
    batch_sweep_vw<VT, MT>(vw, u, op, ranges, nranges, chunks, nchunks, lrow, lfirst, nlong, bs,
                           cs, Yold, Ynew, Zold, Znew, inv_out, P, scratch, part, all_frozen, grid,
                           s, false);
    KNB_CUDA(cudaEventRecord(e1, s));
    KNB_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    KNB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (u == U_CANDIDATES[0] || ms < best_ms) {
      best = u;
      best_ms = ms;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return best;
}

static int vw_for(uint32_t B) {
  if (B <= 32) return 1;
  if (B <= 64) return 2;
  if (B <= 128) return 4;
  return 8;
}

// What batched solves on one operator keep between calls: the row ranges
// and chunks, and every buffer (grown when a call needs more, never shrunk;
// freeing the tens of GB a large batch holds costs as much as a quarter of a
// solve). A solve holds `mu` while it runs, so concurrent calls on one
// operator take turns.
struct BatchWorkspace : Workspace {
  std::mutex mu;
  bool planned = false;
  uint32_t nranges = 0, nchunks = 0, nlong = 0;
  DevBuf<RowRange> d_ranges;
  DevBuf<Chunk> d_chunks;
  DevBuf<uint32_t> d_lrow, d_lfirst, prow, pcols;
  DevBuf<double> pin, dout, Pd, sums, pvals, part, Y64[2], Z64[2], sc64;
  DevBuf<float> Y32[2], Z32[2], sc32;
  DevBuf<ColState> cs;
  DevBuf<int32_t> flags, all_frozen;
};

template <class T>
static void grow(DevBuf<T>& b, size_t count) {
  if (b.n < count) b.alloc(count);
}

void pagerank_batch(GraphHandleImpl& g, const BatchParams& prm, const double* pers_colmajor,
                    double* out_colmajor, BatchInfo* info, cudaStream_t s) {
  const uint32_t n = g.n;
  if (n == 0 || prm.B == 0) return;
  const int which = (g.directed && prm.directed) ? 1 : (g.directed ? 2 : 0);
  const double lfac = prm.loops == 2 ? 0.0 : (which == 1 ? 1.0 : (prm.loops == 0 ? 2.0 : 1.0));
  Operator& op = g.op(which, prm.weighted, lfac, s);
  // arcs in flight per (column width, value types), tuned on first use
  auto tuned_u = [&](int key) {
    std::lock_guard<std::mutex> lock(op.mu);
    auto it = op.batch_u.find(key);
    return it == op.batch_u.end() ? 0 : it->second;
  };
  auto keep_u = [&](int key, int u) {
    std::lock_guard<std::mutex> lock(op.mu);
    op.batch_u[key] = u;
  };
  BatchWorkspace* wsp = nullptr;
  {
    std::lock_guard<std::mutex> lock(op.mu);
    if (!op.batch_ws) op.batch_ws = std::make_unique<BatchWorkspace>();
    wsp = static_cast<BatchWorkspace*>(op.batch_ws.get());
  }
  BatchWorkspace& ws = *wsp;
  std::lock_guard<std::mutex> ws_lock(ws.mu);
  if (!ws.planned) {
    std::vector<uint32_t> hoff(n + 1);
    KNB_CUDA(cudaMemcpyAsync(hoff.data(), op.rows->off.get(), ((size_t)n + 1) * 4,
                             cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    BatchPlan plan = make_plan(hoff, n);
    upload(ws.d_ranges, plan.ranges, s);
    upload(ws.d_chunks, plan.chunks, s);
    upload(ws.d_lrow, plan.lrow, s);
    upload(ws.d_lfirst, plan.lfirst, s);
    ws.nranges = (uint32_t)plan.ranges.size();
    ws.nchunks = (uint32_t)plan.chunks.size();
    ws.nlong = (uint32_t)plan.lrow.size();
    KNB_CUDA(cudaStreamSynchronize(s));
    ws.planned = true;
  }
  const DevBuf<RowRange>& d_ranges = ws.d_ranges;
  const DevBuf<Chunk>& d_chunks = ws.d_chunks;
  const DevBuf<uint32_t>& d_lrow = ws.d_lrow;
  const DevBuf<uint32_t>& d_lfirst = ws.d_lfirst;
  const uint32_t nranges = ws.nranges, nchunks = ws.nchunks, nlong = ws.nlong;
  const unsigned grid = 148 * 4;

  cudaEvent_t t0, t1, l0, l1;
  KNB_CUDA(cudaEventCreate(&t0));
  KNB_CUDA(cudaEventCreate(&t1));
  KNB_CUDA(cudaEventCreate(&l0));
  KNB_CUDA(cudaEventCreate(&l1));
  KNB_CUDA(cudaEventRecord(t0, s));
  double sweep_ms = 0.0;  // device time of the sweep loops alone
  auto loop_end = [&] {
    KNB_CUDA(cudaEventRecord(l1, s));
    KNB_CUDA(cudaEventSynchronize(l1));
    float lm = 0;
    KNB_CUDA(cudaEventElapsedTime(&lm, l0, l1));
    sweep_ms += lm;
  };
  int launches = 0;
  int64_t sweeps32 = 0, sweeps64 = 0, colits32 = 0;
  const bool mixed = prm.precision == PREC_MIXED;
  // mixed: the FP64 phase as one anchor sweep and refinement sweeps (tuning
  // key 9 at 0: plain FP64 sweeps)
  const bool refine = mixed && tuning().refine != 0;
  const uint32_t Btot = prm.B;
  DevBuf<double>& pin = ws.pin;
  grow(pin, (size_t)n * Btot);
  KNB_CUDA(cudaMemcpyAsync(pin.get(), pers_colmajor, (size_t)n * Btot * 8,
                           prm.on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
  double* outp = out_colmajor;
  if (!prm.on_device) {
    grow(ws.dout, (size_t)n * Btot);
    outp = ws.dout.get();
  }
  std::vector<int32_t> col_iters(Btot, 0);
  std::vector<uint8_t> col_conv(Btot, 0);
  // column groups of at most 256
  for (uint32_t c0 = 0; c0 < Btot; c0 += 256) {
    const uint32_t B = std::min<uint32_t>(256, Btot - c0);
    const int vw = vw_for(B);
    DevBuf<double>& Pd = ws.Pd;
    DevBuf<double>& sums = ws.sums;
    DevBuf<double>& pvals = ws.pvals;
    DevBuf<uint32_t>& prow = ws.prow;
    DevBuf<uint32_t>& pcols = ws.pcols;
    DevBuf<int32_t>& flags = ws.flags;
    grow(sums, B);
    grow(prow, (size_t)n + 1);
    grow(flags, 2);
    KNB_CUDA(cudaMemsetAsync(flags.get(), 0, 8, s));
    pers_columns<<<grid_for(B, BW, 1184), BT, 0, s>>>(pin.get() + (size_t)c0 * n, n, B, nullptr,
                                                      flags.get(), sums.get());
    int32_t hf[2];
    KNB_CUDA(cudaMemcpyAsync(hf, flags.get(), 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    if (hf[0] & 1) throw Error("the personalization vector must hold finite, nonnegative values");
    if (hf[0] & 2) throw Error("the personalization vector must have a positive sum");
    // Teleport columns: the nonzero entries per node when at most 1/16 of
    // them are nonzero (seed-set personalisation), else dense; a sweep then
    // reads only the rows that hold seeds.
    KNB_CUDA(cudaMemsetAsync(prow.get(), 0, ((size_t)n + 1) * 4, s));
    pers_row_counts<<<grid_for(n, 256), 256, 0, s>>>(pin.get() + (size_t)c0 * n, n, B, prow.get());
    const uint32_t pnnz = exclusive_scan<uint32_t>(prow.get(), prow.get(), (size_t)n + 1, s);
    PersView P{nullptr, nullptr, nullptr, nullptr};
    if ((uint64_t)pnnz * 16 <= (uint64_t)n * B) {
      grow(pcols, std::max<uint32_t>(pnnz, 1));
      grow(pvals, std::max<uint32_t>(pnnz, 1));
      pers_row_fill<<<grid_for(n, 256), 256, 0, s>>>(pin.get() + (size_t)c0 * n, sums.get(), n, B,
                                                     prow.get(), pcols.get(), pvals.get());
      P = PersView{nullptr, prow.get(), pcols.get(), pvals.get()};
    } else {
      grow(Pd, (size_t)n * B);
      pers_scatter<<<grid_for((uint64_t)n * B, 256), 256, 0, s>>>(pin.get() + (size_t)c0 * n,
                                                                   sums.get(), n, B, Pd.get());
      P = PersView{Pd.get(), nullptr, nullptr, nullptr};
    }
    KNB_LAUNCH("teleport columns");
    launches += 4;
    BatchScalars bs{prm.damping, 1.0 / n, n, B, prm.dangling == 1 ? 1 : 0, 0.0, 0, 0};
    DevBuf<ColState>& cs = ws.cs;
    DevBuf<int32_t>& all_frozen = ws.all_frozen;
    DevBuf<double>& part = ws.part;
    grow(cs, B);
    grow(all_frozen, 1);
    grow(part, std::max<size_t>((size_t)2 * grid * 3 * B, (size_t)1184 * 2 * B));
    const double dterm0 = (double)op.n_dangling / (double)n;
    int64_t done32 = 0;
    const size_t nb = (size_t)n * B;
    DevBuf<float>(&Y32)[2] = ws.Y32;
    DevBuf<float>(&Z32)[2] = ws.Z32;
    DevBuf<float>& sc32 = ws.sc32;
    DevBuf<double>(&Y64)[2] = ws.Y64;
    DevBuf<double>(&Z64)[2] = ws.Z64;
    DevBuf<double>& sc64 = ws.sc64;
    if (mixed) {
      for (int k = 0; k < 2; ++k) {
        grow(Y32[k], nb);
        grow(Z32[k], nb);
      }
      grow(sc32, std::max<size_t>((size_t)nchunks * B, 1));
      spmm_init<float><<<grid_for(nb, 256), 256, 0, s>>>(Y32[0].get(), Z32[0].get(),
                                                          op.inv_out32.get(), n, B, nullptr);
      spmm_set_state<<<1, 256, 0, s>>>(cs.get(), B, dterm0, 0);
      KNB_CUDA(cudaMemsetAsync(all_frozen.get(), 0, 4, s));
      bs.tol = std::max(prm.tol * prm.switch_factor, prm.switch_floor);
      bs.max_iter = (int32_t)prm.max_iter;
      launches += 2;
      int u32 = tuned_u(vw * 4 + 0);
      if (!u32) {
        u32 = tune_arcs_in_flight<float, float>(
            vw, op.view32(), d_ranges, nranges, d_chunks, nchunks, d_lrow, d_lfirst, nlong, bs,
            cs.get(), Y32[0].get(), Y32[1].get(), Z32[0].get(), Z32[1].get(), op.inv_out32.get(),
            P, sc32.get(), part.get(), all_frozen.get(), grid, s);
        keep_u(vw * 4 + 0, u32);
      }
      int k = 0;
      KNB_CUDA(cudaEventRecord(l0, s));
      for (;;) {
        const int b = k & 1;
        launches += batch_sweep_vw<float, float>(
            vw, u32, op.view32(), d_ranges, nranges, d_chunks, nchunks, d_lrow, d_lfirst, nlong,
            bs, cs.get(), Y32[b].get(), Y32[1 - b].get(), Z32[b].get(), Z32[1 - b].get(),
            op.inv_out32.get(), P, sc32.get(), part.get(), all_frozen.get(), grid, s);
        ++k;
        if (k % 4 == 0) {
          int32_t af = 0;
          KNB_CUDA(cudaMemcpyAsync(&af, all_frozen.get(), 4, cudaMemcpyDeviceToHost, s));
          KNB_CUDA(cudaStreamSynchronize(s));
          if (af) break;
        }
      }
      loop_end();
      // every column's FP32 phase ended; hand over from its own buffer
      std::vector<ColState> h(B);
      KNB_CUDA(cudaMemcpyAsync(h.data(), cs.get(), B * sizeof(ColState), cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaStreamSynchronize(s));
      for (uint32_t c = 0; c < B; ++c) {
        if (!h[c].converged)
          throw Error("PageRank did not converge to tolerance " + std::to_string(prm.tol) +
                      " within " + std::to_string(prm.max_iter) + " iterations");
        done32 = std::max<int64_t>(done32, h[c].iter);
      }
      sweeps32 += k;
      // columns stopped at different sweeps: each is read from its own buffer
      for (int kk = 0; kk < 2; ++kk) {
        grow(Y64[kk], nb);
        grow(Z64[kk], nb);
      }
      spmm_switch<<<grid_for(nb, 256), 256, 0, s>>>(Y32[0].get(), Y32[1].get(), cs.get(),
                                                    Y64[0].get(), Z64[0].get(),
                                                    op.inv_out64.get(), n, B);
      column_sums_part<<<1184, 256, 0, s>>>(Y64[0].get(), op.inv_out64.get(), n, B, part.get());
      column_sums_finish<<<1, 256, 0, s>>>(part.get(), 1184, B, cs.get());
      KNB_LAUNCH("batch hand-over");
      launches += 3;
      for (uint32_t c = 0; c < B; ++c) {
        col_iters[c0 + c] = h[c].iter;
        colits32 += h[c].iter;
      }
    } else {
      for (int kk = 0; kk < 2; ++kk) {
        grow(Y64[kk], nb);
        grow(Z64[kk], nb);
      }
      spmm_init<double><<<grid_for(nb, 256), 256, 0, s>>>(Y64[0].get(), Z64[0].get(),
                                                           op.inv_out64.get(), n, B, nullptr);
      spmm_set_state<<<1, 256, 0, s>>>(cs.get(), B, dterm0, 0);
      launches += 2;
    }
    // FP64 phase
    KNB_CUDA(cudaMemsetAsync(all_frozen.get(), 0, 4, s));
    bs.tol = prm.tol;
    bs.max_iter = (int32_t)(prm.max_iter - (mixed ? 0 : 0));
    grow(sc64, std::max<size_t>((size_t)nchunks * B, 1));
    const bool use32v = op.has_vals && op.vals32_exact;
    const int key64 = vw * 4 + (use32v ? 1 : 2);
    int u64 = tuned_u(key64);
    if (!u64) {
      u64 = use32v
                ? tune_arcs_in_flight<double, float>(
                      vw, op.view32(), d_ranges, nranges, d_chunks, nchunks, d_lrow, d_lfirst,
                      nlong, bs, cs.get(), Y64[0].get(), Y64[1].get(), Z64[0].get(), Z64[1].get(),
                      op.inv_out64.get(), P, sc64.get(), part.get(), all_frozen.get(), grid, s)
                : tune_arcs_in_flight<double, double>(
                      vw, op.view64(), d_ranges, nranges, d_chunks, nchunks, d_lrow, d_lfirst,
                      nlong, bs, cs.get(), Y64[0].get(), Y64[1].get(), Z64[0].get(), Z64[1].get(),
                      op.inv_out64.get(), P, sc64.get(), part.get(), all_frozen.get(), grid, s);
      keep_u(key64, u64);
    }
    int k = 0;
    KNB_CUDA(cudaEventRecord(l0, s));
    auto all_done = [&] {
      int32_t af = 0;
      KNB_CUDA(cudaMemcpyAsync(&af, all_frozen.get(), 4, cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaStreamSynchronize(s));
      return af != 0;
    };
    if (refine) {
      // the anchor sweep: FP64 gathers of z_ref = Y64[0] / out; s_ref into
      // Y64[1], the correction e and z_e into Y32[1] and Z32[1]
      const RefineBufs rb0{Y64[0].get(), Y64[1].get(), nullptr, Y32[1].get(), Z32[1].get(),
                           op.inv_out32.get()};
      if (use32v)
        launches += batch_sweep_vw<double, float, EPI_ANCHOR>(
            vw, u64, op.view32(), d_ranges, nranges, d_chunks, nchunks, d_lrow, d_lfirst, nlong,
            bs, cs.get(), Y64[0].get(), Y64[1].get(), Z64[0].get(), Z64[1].get(),
            op.inv_out64.get(), P, sc64.get(), part.get(), all_frozen.get(), grid, s, true, rb0);
      else
        launches += batch_sweep_vw<double, double, EPI_ANCHOR>(
            vw, u64, op.view64(), d_ranges, nranges, d_chunks, nchunks, d_lrow, d_lfirst, nlong,
            bs, cs.get(), Y64[0].get(), Y64[1].get(), Z64[0].get(), Z64[1].get(),
            op.inv_out64.get(), P, sc64.get(), part.get(), all_frozen.get(), grid, s, true, rb0);
      k = 1;
      // refinement sweeps: FP32 gathers of z_e, FP32 arc values (the FP32
      // phase's arcs in flight)
      int ur = tuned_u(vw * 4 + 0);
      if (!ur) ur = 4;
      for (;;) {
        const int b = k & 1;
        const RefineBufs rb{Y64[0].get(), Y64[1].get(), Y32[b].get(), Y32[1 - b].get(),
                            Z32[1 - b].get(), op.inv_out32.get()};
        launches += batch_sweep_vw<float, float, EPI_REFINE>(
            vw, ur, op.view32(), d_ranges, nranges, d_chunks, nchunks, d_lrow, d_lfirst, nlong,
            bs, cs.get(), Y32[b].get(), Y32[1 - b].get(), Z32[b].get(), Z32[1 - b].get(),
            op.inv_out32.get(), P, sc32.get(), part.get(), all_frozen.get(), grid, s, true, rb);
        ++k;
        if (k % 4 == 0 && all_done()) break;
      }
    } else {
      for (;;) {
        const int b = k & 1;
        if (use32v)
          launches += batch_sweep_vw<double, float>(
              vw, u64, op.view32(), d_ranges, nranges, d_chunks, nchunks, d_lrow, d_lfirst, nlong,
              bs, cs.get(), Y64[b].get(), Y64[1 - b].get(), Z64[b].get(), Z64[1 - b].get(),
              op.inv_out64.get(), P, sc64.get(), part.get(), all_frozen.get(), grid, s);
        else
          launches += batch_sweep_vw<double, double>(
              vw, u64, op.view64(), d_ranges, nranges, d_chunks, nchunks, d_lrow, d_lfirst, nlong,
              bs, cs.get(), Y64[b].get(), Y64[1 - b].get(), Z64[b].get(), Z64[1 - b].get(),
              op.inv_out64.get(), P, sc64.get(), part.get(), all_frozen.get(), grid, s);
        ++k;
        if (k % 4 == 0 && all_done()) break;
      }
    }
    loop_end();
    sweeps64 += k;
    std::vector<ColState> h(B);
    KNB_CUDA(cudaMemcpyAsync(h.data(), cs.get(), B * sizeof(ColState), cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    for (uint32_t c = 0; c < B; ++c) {
      if (!h[c].converged)
        throw Error("PageRank did not converge to tolerance " + std::to_string(prm.tol) +
                    " within " + std::to_string(prm.max_iter) + " iterations");
      col_iters[c0 + c] += h[c].iter;
      col_conv[c0 + c] = 1;
    }
    if (refine)
      spmm_output_ref<<<grid_for(nb, 256), 256, 0, s>>>(Y64[0].get(), Y32[0].get(), Y32[1].get(),
                                                        cs.get(), n, B, outp + (size_t)c0 * n);
    else
      spmm_output<double><<<grid_for(nb, 256), 256, 0, s>>>(Y64[0].get(), Y64[1].get(), cs.get(),
                                                            n, B, outp + (size_t)c0 * n);
    ++launches;
  }
  if (!prm.on_device)
    KNB_CUDA(cudaMemcpyAsync(out_colmajor, outp, (size_t)n * Btot * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaEventRecord(t1, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  KNB_CUDA(cudaEventElapsedTime(&ms, t0, t1));
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaEventDestroy(l0);
  cudaEventDestroy(l1);
  if (info) {
    info->seconds = ms * 1e-3;
    info->sweep_seconds = sweep_ms * 1e-3;
    info->sweeps = sweeps32 + sweeps64;
    info->sweeps_fp32 = sweeps32;
    int64_t tot = 0, mx = 0;
    for (uint32_t c = 0; c < Btot; ++c) {
      tot += col_iters[c];
      mx = std::max<int64_t>(mx, col_iters[c]);
    }
    info->column_iterations = tot;
    info->column_iterations_fp32 = colits32;
    info->max_column_iterations = mx;
    info->refined = refine ? 1 : 0;
    info->kernel_launches = launches;
  }
}

}  // namespace knb
