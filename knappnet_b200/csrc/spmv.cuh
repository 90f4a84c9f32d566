// Merge-path sparse matrix-vector product with fused per-row epilogues.
//
// The operator is a row-compressed matrix (row offsets `off`, column indices
// `cols`, optional values `vals`) whose rows list the arcs a measure pulls
// along: for PageRank the arcs arriving at a node (the in-CSR, i.e. the CSC of
// the adjacency matrix), as in the reference's SparseOp
// (crates/engine/src/metrics/eigenvector.rs:498-704).
//
// Work is split by the merge-path decomposition of Merrill and Garland
// (SC'16): the merge of the n row ends with the nnz arcs is cut into tiles of
// TILE = 256 * IPT items, so every CTA does the same amount of work whatever
// the degree distribution (R-MAT hubs with 10^5-10^6 in-arcs included). A CTA
//   1. streams its arcs with coalesced evict-first loads, gathers the iterate
//      with evict-last loads (the iterate is meant to stay in L2), and stages
//      the products in shared memory;
//   2. walks its part of the merge path IPT items per thread, finishing the
//      rows that end inside the tile, and joins the per-thread partial sums of
//      rows that cross threads with a warp segmented scan in a fixed order;
//   3. runs the epilogue (PageRank update, power-iteration shift, plain
//      store) on every row that starts and ends in the tile, and reduces the
//      epilogue's scalars (mass, dangling mass, L1 change, maximum) to one
//      partial per tile.
// Rows that cross a tile boundary ("split rows": hubs, or rows cut by a
// boundary) leave a partial per tile; a second kernel adds them in tile order
// and runs their epilogue, and its last CTA reduces every partial in a fixed
// order. Every sum therefore has a fixed association: results are identical
// from run to run (they differ from the reference's sequential row sums only
// by rounding).
#pragma once

#include "common.cuh"

namespace knb {

constexpr int SPMV_THREADS = 256;

struct TileCoord {
  uint32_t row;  // rows whose end marker precedes this tile
  uint32_t arc;  // arcs consumed before this tile
};

struct SplitRow {
  uint32_t row;    // the row
  uint32_t first;  // tile holding its first arc
  uint32_t last;   // tile that consumes its end marker
};

// Device view of an operator.
template <class MT>
struct OpView {
  uint32_t n;
  uint64_t nnz;
  const uint32_t* off;
  const uint32_t* cols;
  const MT* vals;  // nullptr when every entry is 1
};

// Scalars shared by the kernels of one iteration. Written by the last CTA of
// the split-row kernel (and the exact-change kernel), read by the next sweep.
struct IterState {
  double inv_total;       // 1 / sum of the current (unnormalised) iterate
  double dterm;           // dangling mass of the normalised current iterate
  double prev_inv_total;  // inv_total of the iterate before it
  double total;           // sum of the newest iterate
  double dang;            // its dangling mass
  double change;          // L1 change of the last sweep (see PagerankEpi)
  double tol;             // stopping tolerance of this phase
  double slack;           // |change - exact change| bound used to call K3
  double top;             // power iteration: largest entry of the newest iterate
  int32_t iter;           // sweeps done
  int32_t max_iter;       // sweep cap
  int32_t converged;      // 1 once change <= tol
  int32_t stopped;        // 1 when the cap is reached without convergence
  int32_t ambiguous;      // 1 when the exact change must decide
  uint32_t ticket;        // CTA counter of the last-CTA reductions
  uint32_t ticket2;
  int32_t fault;          // 1 when a sweep gave up waiting for its staged copies
};

__device__ __forceinline__ bool iteration_done(const IterState* st) {
  return st->converged != 0 || st->stopped != 0;
}

// -------------------------------------------------------------------- kernel 1
template <class VT, class MT, class Epi, int IPT>
__global__ void __launch_bounds__(SPMV_THREADS)
tile_spmv(OpView<MT> op, const VT* __restrict__ xg, Epi epi_in,
          const TileCoord* __restrict__ coords, VT* __restrict__ carry, VT* __restrict__ head,
          double* __restrict__ part, const IterState* __restrict__ st) {
  constexpr int T = SPMV_THREADS;
  constexpr int TILE = T * IPT;
  constexpr int NA = Epi::NACC;
  if (st && iteration_done(st)) return;
  Epi epi = epi_in;
  epi.prepare(st);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  VT* prod = reinterpret_cast<VT*>(smem_raw);
  VT* rowsum = prod + TILE;
  VT* cval = rowsum + TILE;
  uint32_t* rend = reinterpret_cast<uint32_t*>(cval + T);
  uint32_t* ckey = rend + TILE + 1;
  __shared__ double red[NA > 0 ? NA : 1][T / 32];
  __shared__ int first_open;

  const uint32_t t = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const uint32_t i0 = coords[t].row, j0 = coords[t].arc;
  const uint32_t i1 = coords[t + 1].row, j1 = coords[t + 1].arc;
  const uint32_t n_rows = i1 - i0, n_arcs = j1 - j0;
  const uint64_t pol_stream = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();

  // 1. products of this tile's arcs: each thread loads IPT arcs strided by T
  //    (coalesced), all index and value loads first, then all gathers, so a
  //    thread keeps IPT independent requests in flight in each phase.
  {
    uint32_t c[IPT];
    VT wv[IPT];
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
      const uint32_t k = tid + q * T;
      c[q] = k < n_arcs ? ld_stream(op.cols + j0 + k, pol_stream) : 0u;
      wv[q] = (op.vals && k < n_arcs) ? (VT)ld_stream(op.vals + j0 + k, pol_stream) : VT(1);
    }
    VT xv[IPT];
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
      const uint32_t k = tid + q * T;
      xv[q] = k < n_arcs ? ld_keep(xg + c[q], pol_keep) : VT(0);
    }
#pragma unroll
    for (int q = 0; q < IPT; ++q) {
      const uint32_t k = tid + q * T;
      if (k < n_arcs) prod[k] = op.vals ? wv[q] * xv[q] : xv[q];
    }
  }
  for (uint32_t r = tid; r < n_rows; r += T) rend[r] = op.off[i0 + r + 1] - j0;
  if (tid == 0) first_open = (i0 < op.n && j0 > op.off[i0]) ? 1 : 0;
  __syncthreads();

  // 2. this thread's IPT items of the merge path
  const uint32_t total = n_rows + n_arcs;
  const uint32_t diag = min((uint32_t)(tid * IPT), total);
  uint32_t lo = diag > n_arcs ? diag - n_arcs : 0, hi = min(diag, n_rows);
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (rend[mid] <= diag - mid - 1) lo = mid + 1; else hi = mid;
  }
  uint32_t ri = lo, aj = diag - lo;
  const uint32_t stop = min(diag + (uint32_t)IPT, total);
  VT acc = VT(0);
#pragma unroll
  for (int it = 0; it < IPT; ++it) {
    if (ri + aj < stop) {
      if (ri < n_rows && aj >= rend[ri]) {
        rowsum[ri] = acc;
        acc = VT(0);
        ++ri;
      } else {
        acc += prod[aj];
        ++aj;
      }
    }
  }
  ckey[tid] = ri;
  cval[tid] = acc;
  __syncthreads();

  // Partial sums of rows that continue past a thread, joined in thread order.
  if (warp == 0) {
    uint32_t pkey = 0xFFFFFFFFu;
    VT pval = VT(0);
    for (int c = 0; c < T / 32; ++c) {
      uint32_t k = ckey[c * 32 + lane];
      VT v = cval[c * 32 + lane];
      if (lane == 0 && k == pkey) v += pval;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t kk = __shfl_up_sync(0xffffffffu, k, o);
        VT vv = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o && kk == k) v += vv;
      }
      uint32_t nxt = __shfl_down_sync(0xffffffffu, k, 1);
      if (lane == 31) nxt = (c + 1 < T / 32) ? ckey[(c + 1) * 32] : 0xFFFFFFFEu;
      if (k != nxt) {
        if (k < n_rows) rowsum[k] += v;
        else carry[t] = v;
      }
      pkey = __shfl_sync(0xffffffffu, k, 31);
      pval = __shfl_sync(0xffffffffu, v, 31);
    }
  }
  __syncthreads();

  // 3. epilogue of the rows that end in this tile
  double a[NA > 0 ? NA : 1];
  Epi::init(a);
  for (uint32_t r = tid; r < n_rows; r += T) {
    if (r == 0 && first_open) {
      head[t] = rowsum[0];
      continue;
    }
    epi.row(i0 + r, rowsum[r], a);
  }
  if constexpr (NA > 0) {
#pragma unroll
    for (int s = 0; s < NA; ++s) {
      double v = Epi::warp_combine(s, a[s]);
      if (lane == 0) red[s][warp] = v;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
      for (int s = 0; s < NA; ++s) {
        double v = lane < T / 32 ? red[s][lane] : Epi::identity(s);
        v = Epi::warp_combine(s, v);
        if (lane == 0) part[(size_t)t * NA + s] = v;
      }
    }
  }
}

// -------------------------------------------------------------------- kernel 1 (warp tiles)
// The same merge-path sweep with one tile per warp (32 * IPT items) and no
// CTA-wide barrier: warps of a CTA share nothing, so a warp waiting for its
// gathers never holds up another and the SM overlaps the phases of its warps.
// Finished row sums stay in registers (indexed by the unrolled item number);
// the partial sums of rows that continue past a lane are joined by one warp
// segmented scan, whose value at lane l-1 is the carry into lane l's first
// finished row.
//
// Products are stored with one pad element after every 128 bytes. Lane l's
// merge-path items start near item l * IPT, so without padding the lanes of
// one read step fall on 32 / IPT banks only; with it, consecutive lanes move
// by IPT + IPT / (128 / sizeof(VT)) elements and spread over all banks, while
// the coalesced writes (item lane + 32 q) stay conflict-free.
template <class VT, int IPT>
struct WarpSmem {
  static constexpr int PAD_SHIFT = sizeof(VT) == 8 ? 4 : 5;
  VT prod[32 * IPT + ((32 * IPT) >> PAD_SHIFT)];
  // tile-relative row ends, at most 32 * IPT: 16 bits keep three 16-warp
  // CTAs of the FP32 sweep under the 100 KB shared-memory carveout, so L1
  // keeps the rest of the SM's 256 KB
  uint16_t rend[32 * IPT + 1];
  static_assert(32 * IPT < 65536, "row ends must fit in 16 bits");
  static __device__ __forceinline__ uint32_t slot(uint32_t k) { return k + (k >> PAD_SHIFT); }
};

// Steps 2-4 of a warp tile once its products are staged in shared memory:
// `prod(a)` is the product of the tile's arc a (0-based), `rend[r]` the
// tile-relative end of row r, `rowbuf` a buffer of at least 32 * IPT values
// that is free once the walk is over (it may alias the products). The
// epilogue's scalars accumulate into this lane's `a` (see
// warp_store_partials).
template <class VT, class Epi, int IPT, class Prod, class RE>
__device__ __forceinline__ void warp_tile_finish(const Prod& prod, VT* rowbuf,
                                                 const RE* rend, uint32_t t, uint32_t i0,
                                                 uint32_t n_rows, uint32_t n_arcs, bool first_open,
                                                 const Epi& epi, VT* __restrict__ carry,
                                                 VT* __restrict__ head, double* a, int lane) {
  // 2. this lane's IPT items of the merge path
  const uint32_t total = n_rows + n_arcs;
  const uint32_t diag = min((uint32_t)(lane * IPT), total);
  uint32_t lo = diag > n_arcs ? diag - n_arcs : 0, hi = min(diag, n_rows);
  while (lo < hi) {
    uint32_t mid = (lo + hi) >> 1;
    if (rend[mid] <= diag - mid - 1) lo = mid + 1; else hi = mid;
  }
  uint32_t ri = lo, aj = diag - lo;
  const uint32_t stop = min(diag + (uint32_t)IPT, total);
  VT acc = VT(0);
  VT fval[IPT];
  uint32_t fmask = 0;  // bit it: item it ended a row
  uint32_t first_row = 0xFFFFFFFFu;
  // end of the current row (kept in a register; 2^32-1 past the last row)
  uint32_t cur_end = ri < n_rows ? rend[ri] : 0xFFFFFFFFu;
#pragma unroll
  for (int it = 0; it < IPT; ++it) {
    fval[it] = VT(0);
    if (ri + aj < stop) {
      if (aj >= cur_end) {
        fval[it] = acc;
        fmask |= 1u << it;
        if (first_row == 0xFFFFFFFFu) first_row = ri;
        acc = VT(0);
        ++ri;
        cur_end = ri < n_rows ? rend[ri] : 0xFFFFFFFFu;
      } else {
        acc += prod(aj);
        ++aj;
      }
    }
  }
  // 3. carries: inclusive segmented scan of (row at lane end, partial). Row
  //    keys never decrease along the lanes, so a lane's segment is the run of
  //    lanes back to the last key change, found once from a ballot; the scan
  //    then only shuffles values.
  const uint32_t key = ri;
  const uint32_t pkey = __shfl_up_sync(0xffffffffu, key, 1);
  const uint32_t starts = __ballot_sync(0xffffffffu, lane == 0 || pkey != key);
  const int seg0 = 31 - __clz(starts & (0xffffffffu >> (31 - lane)));
  VT v = acc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    VT vv = __shfl_up_sync(0xffffffffu, v, o);
    if (lane - o >= seg0) v += vv;
  }
  const VT pval = __shfl_up_sync(0xffffffffu, v, 1);
  const VT cin = (lane > 0 && pkey == first_row) ? pval : VT(0);
  if (lane == 31) carry[t] = v;  // the row open at the tile end (0 if none)

  // 4. epilogue. With IPT >= 8 the finished row sums go to `rowbuf` (a tile
  //    holds at most 32 * IPT rows), then lane l takes rows l, l + 32, ...:
  //    the epilogue runs once per 32 rows, with coalesced accesses to the
  //    per-node vectors, instead of once per item slot. With fewer slots each
  //    lane runs its own rows directly.
  if constexpr (IPT >= 8) {
    __syncwarp();
    uint32_t r = first_row;
#pragma unroll
    for (int it = 0; it < IPT; ++it) {
      if (fmask & (1u << it)) {
        VT sum = fval[it];
        if (r == first_row) sum += cin;
        rowbuf[r] = sum;
        ++r;
      }
    }
    __syncwarp();
    for (uint32_t q = lane; q < n_rows; q += 32) {
      const VT sum = rowbuf[q];
      if (q == 0 && first_open) head[t] = sum;
      else epi.row(i0 + q, sum, a);
    }
  } else {
    uint32_t r = first_row;
#pragma unroll
    for (int it = 0; it < IPT; ++it) {
      if (fmask & (1u << it)) {
        VT sum = fval[it];
        if (r == first_row) sum += cin;
        if (r == 0 && first_open) head[t] = sum;
        else epi.row(i0 + r, sum, a);
        ++r;
      }
    }
  }
}

// One partial per warp: the warp's epilogue scalars (accumulated over all
// its tiles, in tile order per lane) joined over the lanes in a fixed order
// and stored at part[idx * NACC + s].
template <class Epi>
__device__ __forceinline__ void warp_store_partials(const double* a, double* __restrict__ part,
                                                    uint32_t idx, int lane) {
  constexpr int NA = Epi::NACC;
  if constexpr (NA > 0 && NA <= 4 && EpiSums<Epi>::value) {
    const double w = warp_sum_scatter<NA>(a, lane);
    if ((lane & 7) == 0 && (lane >> 3) < NA) part[(size_t)idx * NA + (lane >> 3)] = w;
  } else if constexpr (NA > 0) {
#pragma unroll
    for (int s2 = 0; s2 < NA; ++s2) {
      double w = Epi::warp_combine(s2, a[s2]);
      if (lane == 0) part[(size_t)idx * NA + s2] = w;
    }
  }
}

// Up to 32 bytes of gathered values per lane (8 FP32 or 4 FP64 items) the
// kernel is built for 48 resident warps per SM (at most 42 registers);
// wider tiles keep the registers they need.
template <class VT, int IPT, int WPB>
constexpr int warp_min_blocks() {
  return (IPT * (int)sizeof(VT) <= 32 && 48 / WPB > 0) ? 48 / WPB : 1;
}

// A warp takes tiles t = global warp, + all warps of the grid: launched with
// one warp per tile it does one tile; launched with the CTAs that fit on the
// GPU at once (a persistent grid) it loops, and a launch after convergence
// retires a few thousand CTAs instead of one per tile. Each warp leaves one
// partial of the epilogue's scalars, at part[global warp]: the partials
// number min(warps launched, ntiles).
// GNA: gathers allocate in L1 (0), never (1), or only for columns below
// l1_hot (2), so that the most gathered values stay in L1 while one-off
// gathers pass through.
template <class VT, class MT, class Epi, int IPT, int WPB, int GNA = 0>
__global__ void __launch_bounds__(WPB * 32, (warp_min_blocks<VT, IPT, WPB>()))
warp_spmv(OpView<MT> op, const VT* __restrict__ xg, Epi epi_in,
          const TileCoord* __restrict__ coords, uint32_t ntiles, VT* __restrict__ carry,
          VT* __restrict__ head, double* __restrict__ part, const IterState* __restrict__ st,
          uint32_t l1_hot) {
  using S = WarpSmem<VT, IPT>;
  if (st && iteration_done(st)) return;
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const uint32_t gw = blockIdx.x * WPB + wib;
  uint32_t t = gw;
  if (t >= ntiles) return;
  Epi epi = epi_in;
  epi.prepare(st);
  double acc[Epi::NACC > 0 ? Epi::NACC : 1];
  Epi::init(acc);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  S& sm = reinterpret_cast<S*>(smem_raw)[wib];
  const uint64_t pol_stream = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();
  const uint32_t stride = gridDim.x * WPB;

  for (; t < ntiles; t += stride) {
    const uint32_t i0 = coords[t].row, j0 = coords[t].arc;
    const uint32_t i1 = coords[t + 1].row, j1 = coords[t + 1].arc;
    const uint32_t n_rows = i1 - i0, n_arcs = j1 - j0;

    // 1. products (all index/value loads, then all gathers), row ends
    {
      uint32_t c[IPT];
      VT wv[IPT];
#pragma unroll
      for (int q = 0; q < IPT; ++q) {
        const uint32_t k = lane + q * 32;
        c[q] = k < n_arcs ? ld_stream(op.cols + j0 + k, pol_stream) : 0u;
        wv[q] = (op.vals && k < n_arcs) ? (VT)ld_stream(op.vals + j0 + k, pol_stream) : VT(1);
      }
      VT xv[IPT];
#pragma unroll
      for (int q = 0; q < IPT; ++q) {
        const uint32_t k = lane + q * 32;
        VT x = VT(0);
        if (k < n_arcs) {
          if constexpr (GNA == 1) x = ld_keep_na(xg + c[q], pol_keep);
          else if constexpr (GNA == 2)
            x = c[q] < l1_hot ? ld_keep(xg + c[q], pol_keep) : ld_keep_na(xg + c[q], pol_keep);
          else x = ld_keep(xg + c[q], pol_keep);
        }
        xv[q] = x;
      }
#pragma unroll
      for (int q = 0; q < IPT; ++q) {
        const uint32_t k = lane + q * 32;
        if (k < n_arcs) sm.prod[S::slot(k)] = op.vals ? wv[q] * xv[q] : xv[q];
      }
    }
    for (uint32_t r = lane; r < n_rows; r += 32)
      sm.rend[r] = (uint16_t)(op.off[i0 + r + 1] - j0);
    const bool first_open = i0 < op.n && j0 > op.off[i0];
    __syncwarp();
    warp_tile_finish<VT, Epi, IPT>([&](uint32_t a) { return sm.prod[S::slot(a)]; }, sm.prod,
                                   sm.rend, t, i0, n_rows, n_arcs, first_open, epi, carry, head,
                                   acc, lane);
    __syncwarp();  // the next tile reuses this warp's buffers
  }
  warp_store_partials<Epi>(acc, part, gw, lane);
}

// -------------------------------------------------------------------- kernel 1 (hot-node cache)
// Persistent warp tiles with the most gathered part of the iterate in shared
// memory. Nodes are numbered by decreasing column count (the relabelled
// operator), so x[0, hot_n) holds the values a sweep gathers most: on R-MAT
// scale 24 the first 40,960 nodes take 40% of all gathers. Each CTA (one per
// SM) copies them into shared memory once per launch, and a gather of a
// column below hot_n reads shared memory instead of sending a sector request
// to L2 (the L1-to-L2 request path is what bounds the plain warp kernel).
// Warps then loop over tiles t = global warp, + all warps.
//
// Column indices and values are read with 16-byte loads from the 16-byte
// boundary at or below the tile's first arc, so each 128-byte line a tile
// spans is requested once; the products are staged from that boundary with
// 16-byte shared stores, and 16 bytes of padding after every 128 bytes keep
// both the stores and the merge-path reads free of bank conflicts. The arc
// arrays must be readable up to the next multiple of 4 arcs past the end
// (the relabelled operator's arrays carry that padding).
template <class VT, int IPT>
struct alignas(16) HotWarpSmem {
  static constexpr int GROUP = 16 / (int)sizeof(VT);   // elements per 16 bytes
  static constexpr int ROW = 128 / (int)sizeof(VT);    // elements per 128 bytes
  static constexpr int SPAN = 32 * IPT + 4;            // staged products, lead included
  VT prod[SPAN + (SPAN / ROW + 1) * GROUP];
  uint32_t rend[32 * IPT + 1];
  static __device__ __forceinline__ uint32_t slot(uint32_t k) { return k + (k / ROW) * GROUP; }
};

template <class VT, class MT, class Epi, int IPT, int WPB>
__global__ void __launch_bounds__(WPB * 32, 1)
hot_spmv(OpView<MT> op, const VT* __restrict__ xg, uint32_t hot_n, Epi epi_in,
         const TileCoord* __restrict__ coords, uint32_t ntiles, VT* __restrict__ carry,
         VT* __restrict__ head, double* __restrict__ part, const IterState* __restrict__ st) {
  using S = HotWarpSmem<VT, IPT>;
  constexpr int NV = (8 * IPT + 1 + 31) / 32;  // 16-byte loads per lane per array
  if (st && iteration_done(st)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  S& sm = reinterpret_cast<S*>(smem_raw)[wib];
  VT* hot = reinterpret_cast<VT*>(smem_raw + sizeof(S) * WPB);
  {
    // hot_n is a multiple of 16 / sizeof(VT): whole 16-byte vectors
    const uint4* src = reinterpret_cast<const uint4*>(xg);
    uint4* dst = reinterpret_cast<uint4*>(hot);
    const uint32_t nvec = hot_n / S::GROUP;
    for (uint32_t i = threadIdx.x; i < nvec; i += WPB * 32) dst[i] = __ldg(src + i);
  }
  __syncthreads();
  Epi epi = epi_in;
  epi.prepare(st);
  const uint64_t pol_stream = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();
  const uint32_t gw = blockIdx.x * WPB + wib;
  if (gw >= ntiles) return;
  double acc[Epi::NACC > 0 ? Epi::NACC : 1];
  Epi::init(acc);

  for (uint32_t t = gw; t < ntiles; t += gridDim.x * WPB) {
    const uint32_t i0 = coords[t].row, j0 = coords[t].arc;
    const uint32_t i1 = coords[t + 1].row, j1 = coords[t + 1].arc;
    const uint32_t n_rows = i1 - i0, n_arcs = j1 - j0;
    const uint32_t a0 = j0 & ~3u, lead = j0 - a0;
    // 1. products: every index and value load, then every gather
    {
      uint32_t c[NV][4];
      MT w[NV][4];
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const uint32_t k0 = a0 + 4u * (lane + 32u * q);
        if (k0 < j1) {
          ld_stream4(op.cols + k0, pol_stream, c[q]);
          if (op.vals) ld_stream4(op.vals + k0, pol_stream, w[q]);
        } else {
#pragma unroll
          for (int e = 0; e < 4; ++e) c[q][e] = 0u;
        }
      }
      VT x[NV][4];
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const uint32_t k0 = a0 + 4u * (lane + 32u * q);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const uint32_t k = k0 + e;
          const uint32_t col = c[q][e];
          VT v = VT(0);
          if (k >= j0 && k < j1) {
            if (col < hot_n) v = hot[col];
            else v = ld_keep(xg + col, pol_keep);
          }
          x[q][e] = v;
        }
      }
#pragma unroll
      for (int q = 0; q < NV; ++q) {
        const uint32_t p = 4u * (lane + 32u * q);
        if (a0 + p < j1) {
          VT pr[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) pr[e] = op.vals ? (VT)w[q][e] * x[q][e] : x[q][e];
          VT* dst = sm.prod + S::slot(p);
          if constexpr (sizeof(VT) == 4) {
            *reinterpret_cast<float4*>(dst) = make_float4(pr[0], pr[1], pr[2], pr[3]);
          } else {
            reinterpret_cast<double2*>(dst)[0] = make_double2(pr[0], pr[1]);
            reinterpret_cast<double2*>(dst)[1] = make_double2(pr[2], pr[3]);
          }
        }
      }
    }
    for (uint32_t r = lane; r < n_rows; r += 32) sm.rend[r] = op.off[i0 + r + 1] - j0;
    const bool first_open = i0 < op.n && j0 > op.off[i0];
    __syncwarp();
    warp_tile_finish<VT, Epi, IPT>([&](uint32_t a) { return sm.prod[S::slot(a + lead)]; },
                                   sm.prod, sm.rend, t, i0, n_rows, n_arcs, first_open, epi,
                                   carry, head, acc, lane);
    __syncwarp();  // the next tile reuses this warp's buffers
  }
  warp_store_partials<Epi>(acc, part, gw, lane);
}

template <class VT, int IPT, int WPB>
constexpr size_t hot_warp_smem_bytes() {
  return sizeof(HotWarpSmem<VT, IPT>) * WPB;
}

template <class VT, int IPT, int WPB>
constexpr size_t warp_smem_bytes() {
  return sizeof(WarpSmem<VT, IPT>) * WPB;
}

// Asks for a shared-memory carveout of just what the warp-tile kernel's
// resident CTAs need (their dynamic shared memory and the 1 KB per CTA the
// driver reserves, as a percentage of an SM's 228 KB); the driver rounds the
// hint up to the next configuration it supports and the rest of the SM's
// 256 KB stays L1. Applied once per device.
template <class VT, int IPT, int WPB>
constexpr int warp_fit_carveout() {
  constexpr size_t smem = warp_smem_bytes<VT, IPT, WPB>();
  constexpr int resident = warp_min_blocks<VT, IPT, WPB>();
  constexpr int pct = (int)((resident * (smem + 1024) * 100 + 233471) / 233472) + 1;
  return pct < 100 ? pct : 100;
}

template <class VT, class MT, class Epi, int IPT, int WPB, int GNA = 0>
inline void fit_warp_carveout() {
  set_func_attr((const void*)warp_spmv<VT, MT, Epi, IPT, WPB, GNA>,
                cudaFuncAttributePreferredSharedMemoryCarveout,
                warp_fit_carveout<VT, IPT, WPB>());
}

template <class VT, int IPT>
constexpr size_t tile_smem_bytes() {
  return (size_t)(2 * SPMV_THREADS * IPT + SPMV_THREADS) * sizeof(VT) +
         (size_t)(SPMV_THREADS * IPT + 1 + SPMV_THREADS) * sizeof(uint32_t);
}

// -------------------------------------------------------------------- kernel 2
// Split rows: partials of tiles first..last-1 (carries) plus the head partial
// of tile `last`. Rows spanning few tiles take one thread (carries added in
// tile order); long rows (hubs) take one warp: lane l adds tiles first+l,
// first+l+32, ... in order, then a fixed butterfly joins the lanes. Each CTA
// also reduces a fixed slice of the sweep's `npart` partials (one per tile
// from tile_spmv, one per warp from the warp-tile kernels); the last CTA to
// finish adds the per-CTA results in CTA order and hands them to
// Epi::finish. Every
// sum has a fixed association, so results do not change from run to run.
// Partials written by other CTAs are read with ld.global.cg (L2, not L1).
constexpr int SPLIT_CTAS = 296;

template <class VT, class Epi>
__global__ void __launch_bounds__(SPMV_THREADS)
split_rows(const SplitRow* __restrict__ sr, uint32_t nsr, uint32_t nshort,
           const VT* __restrict__ carry,
           const VT* __restrict__ head, Epi epi_in, const double* __restrict__ part1,
           uint32_t npart, double* __restrict__ part2, IterState* st) {
  constexpr int T = SPMV_THREADS;
  constexpr int NA = Epi::NACC;
  if (st && iteration_done(st)) return;
  Epi epi = epi_in;
  epi.prepare(st);
  __shared__ double red[NA > 0 ? NA : 1][T / 32];
  __shared__ bool last;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double a[NA > 0 ? NA : 1];
  Epi::init(a);
  // short split rows (few tiles): one thread each, carries added in tile order
  for (uint32_t s = blockIdx.x * T + tid; s < nshort; s += gridDim.x * T) {
    const SplitRow r = sr[s];
    VT sum = VT(0);
    for (uint32_t q = r.first; q < r.last; ++q) sum += __ldcg(carry + q);
    sum += __ldcg(head + r.last);
    epi.row(r.row, sum, a);
  }
  // long split rows (hubs): one warp each
  const uint32_t gwarp = blockIdx.x * (T / 32) + warp, nwarps = gridDim.x * (T / 32);
  for (uint32_t s = nshort + gwarp; s < nsr; s += nwarps) {
    const SplitRow r = sr[s];
    VT sum = VT(0);
    for (uint32_t q = r.first + lane; q < r.last; q += 32) sum += __ldcg(carry + q);
    sum = warp_sum(sum);
    if (lane == 0) {
      sum += __ldcg(head + r.last);
      epi.row(r.row, sum, a);
    }
  }
  if constexpr (NA > 0) {
    // this CTA's slice of the sweep's partials, in order per thread
    const uint32_t per = (npart + gridDim.x - 1) / gridDim.x;
    const uint32_t q0 = blockIdx.x * per, q1 = min(npart, q0 + per);
    for (uint32_t q = q0 + tid; q < q1; q += T)
#pragma unroll
      for (int s = 0; s < NA; ++s) a[s] = Epi::combine(s, a[s], __ldcg(part1 + (size_t)q * NA + s));
#pragma unroll
    for (int s = 0; s < NA; ++s) {
      double v = Epi::warp_combine(s, a[s]);
      if (lane == 0) red[s][warp] = v;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
      for (int s = 0; s < NA; ++s) {
        double v = lane < T / 32 ? red[s][lane] : Epi::identity(s);
        v = Epi::warp_combine(s, v);
        if (lane == 0) part2[(size_t)blockIdx.x * NA + s] = v;
      }
    }
  }
  if (st == nullptr) return;
  // last CTA: the per-CTA results in CTA order
  __threadfence();
  __syncthreads();
  if (tid == 0) {
    unsigned int k = atomicAdd(&st->ticket, 1u);
    last = (k == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double tot[NA > 0 ? NA : 1];
#pragma unroll
  for (int s = 0; s < NA; ++s) tot[s] = Epi::identity(s);
  if constexpr (NA > 0) {
    if (warp == 0) {
      for (uint32_t q = lane; q < gridDim.x; q += 32)
#pragma unroll
        for (int s = 0; s < NA; ++s) tot[s] = Epi::combine(s, tot[s], __ldcg(part2 + (size_t)q * NA + s));
#pragma unroll
      for (int s = 0; s < NA; ++s) tot[s] = Epi::warp_combine(s, tot[s]);
    }
  }
  if (tid == 0) {
    epi.finish(st, tot);
    st->ticket = 0;
  }
}

}  // namespace knb
