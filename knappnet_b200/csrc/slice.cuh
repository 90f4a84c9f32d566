// Sliced sparse matrix-vector product with fused per-row epilogues.
//
// The operator is the pull matrix of a measure (for PageRank the arcs
// arriving at each node, the reference's SparseOp,
// crates/engine/src/metrics/eigenvector.rs:498-704) with its nodes
// renumbered by decreasing row length, so rows of one length sit together:
//
// - long rows (at least `lw` arcs) come first, in row-compressed form with
//   each row's arcs sorted by column. Their arcs are cut into pieces of equal
//   size; a warp takes a piece and walks its rows, all 32 lanes reading
//   consecutive arcs of one row (coalesced 128-byte index and value loads;
//   consecutive columns of a hub row often share cache lines of the gathered
//   iterate), and joins the row's lane sums with a fixed butterfly. A row
//   cut by a piece boundary leaves a partial per piece ("carry" for the
//   piece where it continues past the end, "head" for the piece where it
//   ends), added in piece order by split_rows (spmv.cuh).
// - the other rows follow in slices of 32 consecutive rows whose arcs are
//   stored arc-major: arc k of lane l's row at base + 32 k + l. A warp takes
//   a slice, each lane sums its own row sequentially in arc order, and the
//   loads of one arc position are one coalesced 128-byte access. Rows in a
//   slice have (nearly) equal lengths, so lanes rarely idle.
//
// Neither part uses shared memory, so L1 keeps the SM's whole 256 KB for the
// gathers in flight and the most gathered values. The epilogue (PageRank
// update, plain store) runs on every row, with coalesced accesses for the
// slices, and reduces the epilogue's scalars to one partial per warp. Every
// sum has a fixed association, so results are identical from run to run.
#pragma once

#include "spmv.cuh"

namespace knb {

constexpr int SLICE_WPB = 8;  // warps per CTA of the sliced sweep (no shared-memory tier)
constexpr int SLICE_HOT_WPB = 32;  // warps per CTA with the shared-memory tier (one CTA per SM)

// Device view of a sliced operator.
template <class MT>
struct SliceView {
  uint32_t n;          // rows (nodes)
  uint32_t n_long;     // rows [0, n_long) are long
  uint32_t long_arcs;  // arcs of the long rows
  uint32_t piece;      // arcs per piece
  uint32_t npieces;
  uint32_t nslices;    // slices of 32 rows over [n_long, n)
  const uint32_t* loff;   // n_long + 1 offsets of the long rows
  const uint32_t* lcols;  // long_arcs column indices
  const MT* lvals;        // long_arcs values (nullptr: every entry is 1)
  const uint32_t* prow;   // npieces: the row holding each piece's first arc
  const uint32_t* sbase;  // nslices + 1: first element of each slice
  const uint16_t* slen;   // n - n_long row lengths (below lw)
  const uint32_t* scols;  // arc-major slice elements
  const MT* svals;
};

// Gather of the iterate with the L2 keep policy; GNA 2 lets only columns
// below l1_hot allocate in L1 (the most gathered values stay there while
// one-off gathers pass through), GNA 0 allocates every gather. With a
// shared-memory tier (smem non-null) columns below smem_n come from there.
template <int GNA, class VT>
__device__ __forceinline__ VT slice_gather(const VT* xg, uint32_t c, uint32_t l1_hot,
                                           uint64_t pol, const VT* smem = nullptr,
                                           uint32_t smem_n = 0) {
  if (smem != nullptr && c < smem_n) return smem[c];
  if constexpr (GNA == 2) return c < l1_hot ? ld_keep(xg + c, pol) : ld_keep_na(xg + c, pol);
  else return ld_keep(xg + c, pol);
}

// s + w x with one rounding (s + x without values): spelled out so that every
// sliced kernel rounds each arc's term the same way, whatever the compiler
// would contract.
template <class VT, class MT>
__device__ __forceinline__ VT slice_fma(const MT* vals, MT w, VT x, VT s) {
  if (!vals) return s + x;
  if constexpr (sizeof(VT) == 4) return __fmaf_rn((VT)w, x, s);
  else return __fma_rn((VT)w, x, s);
}

// Sum over arcs [lo, hi) of one long row, lanes striding by 32 from the
// 32-arc boundary at or below lo (so each load instruction touches one
// 128-byte line); U arcs per lane in flight; warp butterfly at the end.
template <class VT, class MT, int U, int GNA>
__device__ __forceinline__ VT slice_long_sum(const SliceView<MT>& op, const VT* __restrict__ xg,
                                             uint32_t lo, uint32_t hi, int lane, uint32_t l1_hot,
                                             uint64_t pol_stream, uint64_t pol_keep,
                                             const VT* smem, uint32_t smem_n) {
  VT s = VT(0);
  for (uint32_t k0 = (lo & ~31u) + (uint32_t)lane; k0 < hi; k0 += 32u * U) {
    uint32_t c[U];
    MT w[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t k = k0 + 32u * u;
      const bool ok = k >= lo && k < hi;
      c[u] = ok ? ld_stream(op.lcols + k, pol_stream) : 0u;
      w[u] = (op.lvals && ok) ? ld_stream(op.lvals + k, pol_stream) : MT(0);
    }
    VT x[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const uint32_t k = k0 + 32u * u;
      x[u] = (k >= lo && k < hi) ? slice_gather<GNA>(xg, c[u], l1_hot, pol_keep, smem, smem_n)
                                 : VT(0);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) s = slice_fma<VT, MT>(op.lvals, w[u], x[u], s);
  }
  return warp_sum(s);
}

// One sweep: every warp first takes pieces t = global warp, + all warps,
// then slices the same way, and leaves one partial of the epilogue's
// scalars at part[global warp] (all warps of the grid write one). With
// smem_n > 0 each CTA first copies x[0, smem_n) (the most gathered values;
// smem_n a multiple of 16 / sizeof(VT)) into shared memory, and gathers of
// those columns read it there instead of sending a request to L1 and L2.
template <class VT, class MT, class Epi, int U, int WPB, int MINB, int GNA>
__global__ void __launch_bounds__(WPB * 32, MINB)
slice_spmv(SliceView<MT> op, const VT* __restrict__ xg, Epi epi_in, VT* __restrict__ carry,
           VT* __restrict__ head, double* __restrict__ part, const IterState* __restrict__ st,
           uint32_t l1_hot, uint32_t smem_n) {
  if (st && iteration_done(st)) return;
  extern __shared__ __align__(16) unsigned char slice_smem[];
  const VT* hot = nullptr;
  if (smem_n > 0) {
    const uint4* src = reinterpret_cast<const uint4*>(xg);
    uint4* dst = reinterpret_cast<uint4*>(slice_smem);
    const uint32_t nvec = smem_n * (uint32_t)sizeof(VT) / 16u;
    for (uint32_t i = threadIdx.x; i < nvec; i += WPB * 32) dst[i] = __ldg(src + i);
    __syncthreads();
    hot = reinterpret_cast<const VT*>(slice_smem);
  }
  constexpr bool EARLY = sizeof(VT) == 4;
  const int lane = threadIdx.x & 31;
  const uint32_t gw = blockIdx.x * WPB + (threadIdx.x >> 5);
  const uint32_t nw = gridDim.x * WPB;
  Epi epi = epi_in;
  epi.prepare(st);
  double acc[Epi::NACC > 0 ? Epi::NACC : 1];
  Epi::init(acc);
  const uint64_t pol_stream = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();

  // long rows, piece by piece
  for (uint32_t t = gw; t < op.npieces; t += nw) {
    const uint32_t a0 = t * op.piece;
    const uint32_t a1 = min(a0 + op.piece, op.long_arcs);
    uint32_t r = op.prow[t];
    uint32_t rs = op.loff[r], re = op.loff[r + 1];
    while (true) {
      // FP32 sweeps load the epilogue's inputs before the row sum (3% faster
      // on R-MAT 24); FP64 sweeps, short of registers, load them after it
      typename Epi::In ein{};
      if (EARLY && lane == 0 && rs >= a0 && re <= a1) ein = epi.fetch(r);
      const VT sum = slice_long_sum<VT, MT, U, GNA>(op, xg, max(rs, a0), min(re, a1), lane,
                                                    l1_hot, pol_stream, pol_keep, hot, smem_n);
      if (re > a1) {  // continues in the next piece
        if (lane == 0) carry[t] = sum;
        break;
      }
      if (rs < a0) {  // began in an earlier piece, ends here
        if (lane == 0) head[t] = sum;
      } else if (lane == 0) {
        if (EARLY) epi.row_in(r, sum, ein, acc);
        else epi.row(r, sum, acc);
      }
      if (re == a1) break;
      ++r;
      rs = re;
      re = op.loff[r + 1];
    }
  }

  // short rows, slice by slice: lane l sums row n_long + 32 s + l in arc order
  for (uint32_t sl = gw; sl < op.nslices; sl += nw) {
    const uint32_t r = op.n_long + sl * 32u + (uint32_t)lane;
    const uint32_t len = r < op.n ? (uint32_t)op.slen[r - op.n_long] : 0u;
    const uint32_t lmax = __shfl_sync(0xffffffffu, len, 0);  // rows descend in length
    const uint32_t base = op.sbase[sl] + (uint32_t)lane;
    typename Epi::In ein{};
    if (EARLY && r < op.n) ein = epi.fetch(r);
    VT s = VT(0);
    for (uint32_t k0 = 0; k0 < lmax; k0 += U) {
      uint32_t c[U];
      MT w[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint32_t k = k0 + u;
        const bool ok = k < len;
        c[u] = ok ? ld_stream(op.scols + base + 32u * k, pol_stream) : 0u;
        w[u] = (op.svals && ok) ? ld_stream(op.svals + base + 32u * k, pol_stream) : MT(0);
      }
      VT x[U];
#pragma unroll
      for (int u = 0; u < U; ++u)
        x[u] = (k0 + u < len) ? slice_gather<GNA>(xg, c[u], l1_hot, pol_keep, hot, smem_n)
                              : VT(0);
#pragma unroll
      for (int u = 0; u < U; ++u) s = slice_fma<VT, MT>(op.svals, w[u], x[u], s);
    }
    if (r < op.n) {
      if (EARLY) epi.row_in(r, s, ein, acc);
      else epi.row(r, s, acc);
    }
  }
  warp_store_partials<Epi>(acc, part, gw, lane);
}

}  // namespace knb
