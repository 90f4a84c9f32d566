// Sliced sweep with its arc streams staged in shared memory by the bulk-copy
// (TMA) engine.
//
// Same operator, work split and arithmetic as slice_spmv (slice.cuh): warps
// take long-row pieces, then slices of 32 short rows; every lane adds the
// same arcs in the same order and long rows join their lanes with the same
// butterfly, so the results are bit-identical to slice_spmv's. What changes
// is how the column and value streams reach the warp. In slice_spmv a lane
// loads its columns from HBM and only then gathers the iterate, so every
// group of arcs waits for two memory latencies back to back. Here each warp
// owns a ring of S shared-memory stages; lane 0 hands the copy engine
// `cp.async.bulk` copies of the warp's next chunks (32 U arcs of columns and
// values, contiguous in both layouts) S - 1 chunks ahead, each completing on
// the stage's mbarrier. The lanes read columns from shared memory and issue
// their gathers at once: the stream latency leaves the warp's critical path
// and the registers stay free for gathers in flight.
//
// Every wait is bounded (about one second of SM clock). A wait that runs out
// marks the sweep's state (fault, stopped) and the warp stops taking work
// after a bounded wait for the copies it still has in flight; the host turns
// the mark into an error. For the test of that path the host can name one
// chunk of the grid's first warp whose copies are never issued (skip_chunk),
// so its wait runs out.
#pragma once

#include "slice.cuh"

namespace knb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Makes barrier initialisation visible to the copy engine.
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrives on the barrier and expects `bytes` of copies to complete on it.
__device__ __forceinline__ void mbar_expect(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Waits for the barrier's phase of parity `parity` for at most `limit` SM
// clock cycles; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, long long limit) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity))
    if (clock64() - t0 > limit) return false;
  return true;
}

// Global to shared copy of `bytes` (a multiple of 16, both addresses 16-byte
// aligned) completing on `bar`, with an L2 eviction policy for the source.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes,
                                         uint32_t bar, uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint "
      "[%0], [%1], %2, [%3], %4;" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar), "l"(pol)
      : "memory");
}

constexpr long long BULK_WAIT_CYCLES = 2000000000ll;  // about one second
constexpr long long BULK_DRAIN_CYCLES = 200000000ll;  // after a fault, per stage
constexpr uint32_t BULK_NO_SKIP = 0xFFFFFFFFu;

// Bytes of one warp's ring: S stages of 32 U columns and 32 U values, then S
// barriers, rounded to 128 bytes.
template <class MT, int U, int S>
__host__ __device__ constexpr uint32_t bulk_ring_bytes() {
  return (uint32_t)((S * 32 * U * (4 + sizeof(MT)) + 8 * S + 127) / 128 * 128);
}

// The chunk sequence of one warp: the chunks of its pieces (t = gw, gw + nw,
// ...; 32 U arcs from the 32-arc boundary at or below the piece's first arc
// up to its last arc rounded up to 32), then the chunks of its slices (U
// arc positions of 32 lanes each). The producer walks it one chunk ahead of
// every issue; the consumer's loops visit the same chunks in the same order.
template <class MT, int U>
struct BulkCursor {
  uint32_t kind;  // 0 long pieces, 1 slices, 2 done
  uint32_t item;  // piece or slice
  uint32_t pos;   // long: first arc of the chunk; slices: first arc position
  uint32_t end;   // long: last arc of the piece rounded up to 32; slices: width
  uint32_t base;  // slices: first element of the slice

  __device__ __forceinline__ void set_item(const SliceView<MT>& op) {
    if (kind == 0) {
      const uint32_t a0 = item * op.piece;
      const uint32_t a1 = min(a0 + op.piece, op.long_arcs);
      pos = a0 & ~31u;
      end = (a1 + 31u) & ~31u;
    } else {
      base = op.sbase[item];
      pos = 0;
      end = (op.sbase[item + 1] - base) >> 5;
    }
  }
  // Moves to the first item at or after the current one that has a chunk.
  __device__ __forceinline__ void settle(const SliceView<MT>& op, uint32_t gw, uint32_t nw) {
    while (kind < 2) {
      const uint32_t count = kind == 0 ? op.npieces : op.nslices;
      if (item >= count) {
        ++kind;
        item = gw;
        continue;
      }
      set_item(op);
      if (pos < end) return;
      item += nw;
    }
  }
  __device__ __forceinline__ void start(const SliceView<MT>& op, uint32_t gw, uint32_t nw) {
    kind = 0;
    item = gw;
    settle(op, gw, nw);
  }
  __device__ __forceinline__ void next(const SliceView<MT>& op, uint32_t gw, uint32_t nw) {
    pos += kind == 0 ? 32u * U : (uint32_t)U;
    if (pos < end) return;
    item += nw;
    settle(op, gw, nw);
  }
  // Issues the copies of the current chunk into a stage (lane 0 only).
  __device__ __forceinline__ void issue(const SliceView<MT>& op, uint32_t cols_dst,
                                        uint32_t vals_dst, uint32_t bar, uint64_t pol) const {
    const uint32_t arcs = kind == 0 ? min(32u * U, end - pos) : 32u * min((uint32_t)U, end - pos);
    const size_t first = kind == 0 ? (size_t)pos : (size_t)base + 32u * (size_t)pos;
    const uint32_t* cs = kind == 0 ? op.lcols : op.scols;
    const MT* vs = kind == 0 ? op.lvals : op.svals;
    const uint32_t cb = arcs * 4u;
    const uint32_t vb = vs ? arcs * (uint32_t)sizeof(MT) : 0u;
    mbar_expect(bar, cb + vb);
    bulk_g2s(cols_dst, cs + first, cb, bar, pol);
    if (vs) bulk_g2s(vals_dst, vs + first, vb, bar, pol);
  }
};

// One warp's ring of stages in dynamic shared memory.
template <class MT, int U, int S>
struct BulkRing {
  uint32_t* cols;  // S stages of 32 U columns
  MT* vals;        // S stages of 32 U values
  uint32_t bar0;   // shared address of the first of S barriers

  __device__ __forceinline__ BulkRing(unsigned char* base) {
    cols = reinterpret_cast<uint32_t*>(base);
    vals = reinterpret_cast<MT*>(base + S * 32 * U * 4);
    bar0 = smem_u32(base + S * 32 * U * (4 + sizeof(MT)));
  }
  __device__ __forceinline__ uint32_t bar(uint32_t j) const { return bar0 + 8u * j; }
  __device__ __forceinline__ uint32_t cols_at(uint32_t j) const {
    return smem_u32(cols + j * 32u * U);
  }
  __device__ __forceinline__ uint32_t vals_at(uint32_t j) const {
    return smem_u32(vals + j * 32u * U);
  }
};

// Per-warp pipeline state: chunks issued and consumed, and whether a wait ran
// out. Lane 0 issues; every lane waits.
template <class MT, int U, int S>
struct BulkPipe {
  BulkRing<MT, U, S> ring;
  BulkCursor<MT, U> prod;
  uint32_t issued = 0, used = 0;
  bool failed = false;

  __device__ __forceinline__ BulkPipe(unsigned char* base) : ring(base) {}

  uint32_t skip = BULK_NO_SKIP;  // a chunk never issued (the wait-limit test)

  __device__ __forceinline__ void issue_one(const SliceView<MT>& op, int lane, uint32_t gw,
                                            uint32_t nw, uint64_t pol) {
    const uint32_t j = issued % S;
    if (lane == 0 && issued != skip)
      prod.issue(op, ring.cols_at(j), ring.vals_at(j), ring.bar(j), pol);
    ++issued;
    prod.next(op, gw, nw);
  }
  // Waits for the next chunk; its stage index, or -1 after a fault (the
  // whole warp agrees, so lanes never part at a warp barrier).
  __device__ __forceinline__ int acquire() {
    const uint32_t j = used % S;
    const uint32_t parity = (used / S) & 1u;
    const bool ok = mbar_wait_bounded(ring.bar(j), parity, BULK_WAIT_CYCLES);
    if (!__all_sync(0xffffffffu, ok)) {
      failed = true;
      return -1;
    }
    return (int)j;
  }
  // The chunk's stage is read: refill it with the chunk S ahead.
  __device__ __forceinline__ void release(const SliceView<MT>& op, int lane, uint32_t gw,
                                          uint32_t nw, uint64_t pol) {
    ++used;
    __syncwarp();
    if (prod.kind < 2) issue_one(op, lane, gw, nw, pol);
  }
  // After a fault: bounded waits for every copy still in flight.
  __device__ __forceinline__ void drain() {
    for (; used < issued; ++used)
      mbar_wait_bounded(ring.bar(used % S), (used / S) & 1u, BULK_DRAIN_CYCLES);
  }
};

// The sweep. Warps per CTA WPB, MINB CTAs per SM; dynamic shared memory:
// WPB rings of bulk_ring_bytes<MT, U, S>().
template <class VT, class MT, class Epi, int U, int S, int WPB, int MINB, int GNA>
__global__ void __launch_bounds__(WPB * 32, MINB)
slice_bulk_spmv(SliceView<MT> op, const VT* __restrict__ xg, Epi epi_in, VT* __restrict__ carry,
                VT* __restrict__ head, double* __restrict__ part, IterState* __restrict__ st,
                uint32_t l1_hot, uint32_t skip_chunk) {
  if (st && iteration_done(st)) return;
  extern __shared__ __align__(128) unsigned char bulk_smem[];
  constexpr bool EARLY = sizeof(VT) == 4;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const uint32_t gw = blockIdx.x * WPB + (uint32_t)wib;
  const uint32_t nw = gridDim.x * WPB;
  Epi epi = epi_in;
  epi.prepare(st);
  double acc[Epi::NACC > 0 ? Epi::NACC : 1];
  Epi::init(acc);
  const uint64_t pol_stream = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();

  BulkPipe<MT, U, S> pipe(bulk_smem + (size_t)wib * bulk_ring_bytes<MT, U, S>());
  if (gw == 0) pipe.skip = skip_chunk;
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < S; ++j) mbar_init(pipe.ring.bar(j), 1);
    mbar_fence_init();
  }
  __syncwarp();
  pipe.prod.start(op, gw, nw);
  for (int j = 0; j < S && pipe.prod.kind < 2; ++j) pipe.issue_one(op, lane, gw, nw, pol_stream);

  // long rows, piece by piece
  for (uint32_t t = gw; t < op.npieces && !pipe.failed; t += nw) {
    const uint32_t a0 = t * op.piece;
    const uint32_t a1 = min(a0 + op.piece, op.long_arcs);
    const uint32_t r1 = (a1 + 31u) & ~31u;
    uint32_t r = op.prow[t];
    uint32_t rs = op.loff[r], re = op.loff[r + 1];
    typename Epi::In ein{};
    if (EARLY && lane == 0 && rs >= a0 && re <= a1) ein = epi.fetch(r);
    VT s = VT(0);
    bool done = false;  // the piece's last row has ended
    for (uint32_t A = a0 & ~31u; A < r1; A += 32u * U) {
      const int j = pipe.acquire();
      if (j < 0) break;
      const uint32_t steps = min((uint32_t)U, (r1 - A) >> 5);
      VT x[U];
      MT w[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const uint32_t k = A + 32u * u + (uint32_t)lane;
        const bool ok = (uint32_t)u < steps && k >= a0 && k < a1;
        const uint32_t c = ok ? pipe.ring.cols[j * 32 * U + 32 * u + lane] : 0u;
        w[u] = (op.lvals && ok) ? pipe.ring.vals[j * 32 * U + 32 * u + lane] : MT(0);
        x[u] = ok ? slice_gather<GNA>(xg, c, l1_hot, pol_keep) : VT(0);
      }
      pipe.release(op, lane, gw, nw, pol_stream);
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if ((uint32_t)u >= steps || done) break;
        const uint32_t kb = A + 32u * u;
        const uint32_t k = kb + (uint32_t)lane;
        const uint32_t step_end = min(kb + 32u, a1);
        while (true) {
          if (k >= rs && k < re) s = slice_fma<VT, MT>(op.lvals, w[u], x[u], s);
          if (re > step_end) break;  // row r continues after this step
          const VT sum = warp_sum(s);
          s = VT(0);
          if (rs < a0) {
            if (lane == 0) head[t] = sum;
          } else if (lane == 0) {
            if (EARLY) epi.row_in(r, sum, ein, acc);
            else epi.row(r, sum, acc);
          }
          if (re >= a1) {
            done = true;
            break;
          }
          ++r;
          rs = re;
          re = op.loff[r + 1];
          if (EARLY && lane == 0 && re <= a1) ein = epi.fetch(r);
        }
      }
    }
    if (!done && !pipe.failed) {  // the last row continues in the next piece
      const VT sum = warp_sum(s);
      if (lane == 0) carry[t] = sum;
    }
  }

  // short rows, slice by slice: lane l sums row n_long + 32 s + l in arc order
  for (uint32_t sl = gw; sl < op.nslices && !pipe.failed; sl += nw) {
    const uint32_t r = op.n_long + sl * 32u + (uint32_t)lane;
    const uint32_t len = r < op.n ? (uint32_t)op.slen[r - op.n_long] : 0u;
    const uint32_t width = (op.sbase[sl + 1] - op.sbase[sl]) >> 5;
    typename Epi::In ein{};
    if (EARLY && r < op.n) ein = epi.fetch(r);
    VT s = VT(0);
    for (uint32_t k0 = 0; k0 < width; k0 += U) {
      const int j = pipe.acquire();
      if (j < 0) break;
      VT x[U];
      MT w[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool ok = k0 + u < len;  // len <= width
        const uint32_t c = ok ? pipe.ring.cols[j * 32 * U + 32 * u + lane] : 0u;
        w[u] = (op.svals && ok) ? pipe.ring.vals[j * 32 * U + 32 * u + lane] : MT(0);
        x[u] = ok ? slice_gather<GNA>(xg, c, l1_hot, pol_keep) : VT(0);
      }
      pipe.release(op, lane, gw, nw, pol_stream);
#pragma unroll
      for (int u = 0; u < U; ++u) s = slice_fma<VT, MT>(op.svals, w[u], x[u], s);
    }
    if (r < op.n && !pipe.failed) {
      if (EARLY) epi.row_in(r, s, ein, acc);
      else epi.row(r, s, acc);
    }
  }
  if (pipe.failed) {
    pipe.drain();
    if (lane == 0 && st) {
      atomicExch(&st->fault, 1);
      atomicExch(&st->stopped, 1);
    }
  }
  __syncwarp();
  warp_store_partials<Epi>(acc, part, gw, lane);
}

}  // namespace knb
