// Device graph build: validation, stable CSR construction by LSD radix sort,
// undirected arc expansion, degree/strength, and the operators of the
// spectral measures.
#include <algorithm>
#include <cstring>

#include "graph.cuh"

namespace knb {

cudaStream_t thread_stream() {
  thread_local cudaStream_t s = nullptr;
  thread_local int dev = -1;
  int cur = 0;
  KNB_CUDA(cudaGetDevice(&cur));
  if (s == nullptr || dev != cur) {
    KNB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    dev = cur;
  }
  return s;
}

// ======================================================================= scan
constexpr int SCAN_T = 256, SCAN_IPT = 16, SCAN_TILE = SCAN_T * SCAN_IPT;

template <class T>
__global__ void scan_reduce(const T* __restrict__ in, size_t n, T* __restrict__ sums) {
  __shared__ T sh[SCAN_T / 32];
  size_t base = (size_t)blockIdx.x * SCAN_TILE;
  T acc = 0;
  for (int k = threadIdx.x; k < SCAN_TILE; k += SCAN_T) {
    size_t i = base + k;
    if (i < n) acc += in[i];
  }
  acc = block_sum(acc, sh);
  if (threadIdx.x == 0) sums[blockIdx.x] = acc;
}

// Exclusive scan of one tile held in shared memory; `carry_in` is added.
template <class T>
__device__ T block_exclusive_scan_tile(T* tile, T carry_in) {
  __shared__ T wsum[SCAN_T / 32];
  int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  T v[SCAN_IPT];
  T run = 0;
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) {
    v[k] = tile[tid * SCAN_IPT + k];
    T x = v[k];
    v[k] = run;
    run += x;
  }
  // inclusive warp scan of thread totals
  T incl = run;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    T x = lane < SCAN_T / 32 ? wsum[lane] : T(0);
    T xi = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      T y = __shfl_up_sync(0xffffffffu, xi, o);
      if (lane >= o) xi += y;
    }
    if (lane < SCAN_T / 32) wsum[lane] = xi - x;  // exclusive
  }
  __syncthreads();
  T offset = carry_in + wsum[w] + (incl - run);
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) tile[tid * SCAN_IPT + k] = v[k] + offset;
  __syncthreads();
  T total = 0;
  if (tid == SCAN_T - 1) total = offset + run;  // only meaningful on the last thread
  return total;
}

template <class T>
__global__ void scan_down(const T* in, T* out, size_t n, const T* __restrict__ sums) {
  __shared__ T tile[SCAN_TILE];
  size_t base = (size_t)blockIdx.x * SCAN_TILE;
  for (int k = threadIdx.x; k < SCAN_TILE; k += SCAN_T) {
    size_t i = base + k;
    tile[k] = i < n ? in[i] : T(0);
  }
  __syncthreads();
  block_exclusive_scan_tile<T>(tile, sums[blockIdx.x]);
  for (int k = threadIdx.x; k < SCAN_TILE; k += SCAN_T) {
    size_t i = base + k;
    if (i < n) out[i] = tile[k];
  }
}

// One CTA scans the per-tile sums in place (chunks of one tile, carried).
template <class T>
__global__ void scan_sums(T* sums, size_t nb, T* total) {
  __shared__ T tile[SCAN_TILE];
  __shared__ T carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (size_t base = 0; base < nb; base += SCAN_TILE) {
    for (int k = threadIdx.x; k < SCAN_TILE; k += SCAN_T)
      tile[k] = base + k < nb ? sums[base + k] : T(0);
    __syncthreads();
    T c = carry;
    __syncthreads();
    T t = block_exclusive_scan_tile<T>(tile, c);
    for (int k = threadIdx.x; k < SCAN_TILE; k += SCAN_T)
      if (base + k < nb) sums[base + k] = tile[k];
    if (threadIdx.x == SCAN_T - 1) carry = t;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total = carry;
}

template <class T>
T exclusive_scan(const T* in, T* out, size_t n, cudaStream_t s) {
  if (n == 0) return 0;
  size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  DevBuf<T> sums(nb + 1);
  scan_reduce<T><<<(unsigned)nb, SCAN_T, 0, s>>>(in, n, sums.get());
  KNB_LAUNCH("scan_reduce");
  scan_sums<T><<<1, SCAN_T, 0, s>>>(sums.get(), nb, sums.get() + nb);
  KNB_LAUNCH("scan_sums");
  scan_down<T><<<(unsigned)nb, SCAN_T, 0, s>>>(in, out, n, sums.get());
  KNB_LAUNCH("scan_down");
  T total = 0;
  KNB_CUDA(cudaMemcpyAsync(&total, sums.get() + nb, sizeof(T), cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  return total;
}
template uint32_t exclusive_scan<uint32_t>(const uint32_t*, uint32_t*, size_t, cudaStream_t);
template uint64_t exclusive_scan<uint64_t>(const uint64_t*, uint64_t*, size_t, cudaStream_t);

// ======================================================================= radix sort
// Stable LSD radix sort of 64-bit keys with a 32-bit payload, 8 bits a pass.
// Stability inside a tile comes from ranking elements warp by warp in input
// order (__match_any_sync groups equal digits of a round), so equal keys keep
// their input order, exactly like the reference's stable counting sorts.
constexpr int RS_T = 256, RS_IPT = 8, RS_TILE = RS_T * RS_IPT;

__global__ void radix_hist(const uint64_t* __restrict__ keys, size_t n, int shift,
                           uint32_t* __restrict__ hist, uint32_t ntiles) {
  __shared__ uint32_t cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  size_t base = (size_t)blockIdx.x * RS_TILE;
  for (int k = threadIdx.x; k < RS_TILE; k += RS_T) {
    size_t i = base + k;
    if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  hist[(size_t)threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

__global__ void radix_scatter(const uint64_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                              uint64_t* __restrict__ kout, uint32_t* __restrict__ vout, size_t n,
                              int shift, const uint32_t* __restrict__ offs, uint32_t ntiles) {
  __shared__ uint32_t wcount[RS_T / 32][256];
  __shared__ uint32_t base_d[256];
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  for (int d = lane; d < 256; d += 32) wcount[w][d] = 0;
  __syncwarp();
  const size_t wbase = (size_t)blockIdx.x * RS_TILE + (size_t)w * 32 * RS_IPT;
  uint64_t key[RS_IPT];
  uint32_t val[RS_IPT], rank[RS_IPT], dig[RS_IPT];
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int r = 0; r < RS_IPT; ++r) {
    size_t i = wbase + (size_t)r * 32 + lane;
    bool ok = i < n;
    key[r] = ok ? kin[i] : 0;
    val[r] = ok ? vin[i] : 0;
    uint32_t d = ok ? (uint32_t)((key[r] >> shift) & 255u) : 256u;
    dig[r] = d;
    uint32_t peers = __match_any_sync(0xffffffffu, d);
    uint32_t before = __popc(peers & lt);
    uint32_t seen = ok ? wcount[w][d] : 0;
    rank[r] = seen + before;
    __syncwarp();
    if (ok && before == 0) wcount[w][d] = seen + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  {
    int d = tid;  // one digit per thread (256 threads)
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < RS_T / 32; ++ww) {
      uint32_t c = wcount[ww][d];
      wcount[ww][d] = run;
      run += c;
    }
    base_d[d] = offs[(size_t)d * ntiles + blockIdx.x];
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < RS_IPT; ++r) {
    size_t i = wbase + (size_t)r * 32 + lane;
    if (i < n) {
      uint32_t d = dig[r];
      size_t pos = (size_t)base_d[d] + wcount[w][d] + rank[r];
      kout[pos] = key[r];
      vout[pos] = val[r];
    }
  }
}

// Sorts (keys, vals) by the low `bits` bits of the keys; the result ends in
// (keys, vals) again. Scratch of the same size is used for the ping-pong.
void radix_sort(uint64_t* keys, uint32_t* vals, size_t n, int bits, cudaStream_t s) {
  if (n <= 1 || bits <= 0) return;
  uint32_t ntiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
  DevBuf<uint64_t> k2(n);
  DevBuf<uint32_t> v2(n);
  DevBuf<uint32_t> hist((size_t)256 * ntiles);
  uint64_t* ka = keys;
  uint32_t* va = vals;
  uint64_t* kb = k2.get();
  uint32_t* vb = v2.get();
  int passes = (bits + 7) / 8;
  for (int p = 0; p < passes; ++p) {
    int shift = 8 * p;
    radix_hist<<<ntiles, RS_T, 0, s>>>(ka, n, shift, hist.get(), ntiles);
    KNB_LAUNCH("radix_hist");
    exclusive_scan<uint32_t>(hist.get(), hist.get(), (size_t)256 * ntiles, s);
    radix_scatter<<<ntiles, RS_T, 0, s>>>(ka, va, kb, vb, n, shift, hist.get(), ntiles);
    KNB_LAUNCH("radix_scatter");
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    KNB_CUDA(cudaMemcpyAsync(keys, ka, n * 8, cudaMemcpyDeviceToDevice, s));
    KNB_CUDA(cudaMemcpyAsync(vals, va, n * 4, cudaMemcpyDeviceToDevice, s));
  }
  KNB_CUDA(cudaStreamSynchronize(s));
}

static int bits_for(uint64_t n) {
  int b = 0;
  while (b < 64 && (1ull << b) < n) ++b;
  return b;
}

// ======================================================================= CSR build
__global__ void make_keys(const uint32_t* __restrict__ from, const uint32_t* __restrict__ to,
                          const uint32_t* __restrict__ edge, uint64_t arcs, int tbits,
                          uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < arcs;
       k += (uint64_t)gridDim.x * blockDim.x) {
    keys[k] = ((uint64_t)from[k] << tbits) | to[k];
    vals[k] = edge ? edge[k] : (uint32_t)k;
  }
}

__global__ void split_keys(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                           uint64_t arcs, int tbits, const double* __restrict__ edge_w,
                           uint32_t* __restrict__ tgt, uint32_t* __restrict__ eidx,
                           double* __restrict__ w) {
  const uint64_t mask = (tbits >= 64) ? ~0ull : ((1ull << tbits) - 1);
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < arcs;
       k += (uint64_t)gridDim.x * blockDim.x) {
    tgt[k] = (uint32_t)(keys[k] & mask);
    uint32_t e = vals[k];
    eidx[k] = e;
    if (w) w[k] = edge_w[e];
  }
}

// off[v] = first sorted arc whose source is >= v (boundaries of the rows).
__global__ void row_bounds(const uint64_t* __restrict__ keys, uint64_t arcs, int tbits,
                           uint32_t n, uint32_t* __restrict__ off) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k <= arcs;
       k += (uint64_t)gridDim.x * blockDim.x) {
    int64_t prev = k == 0 ? -1 : (int64_t)(keys[k - 1] >> tbits);
    int64_t cur = k == arcs ? (int64_t)n : (int64_t)(keys[k] >> tbits);
    for (int64_t v = prev + 1; v <= cur; ++v) off[v] = (uint32_t)k;
  }
}

void build_csr(uint32_t n, uint64_t arcs, const uint32_t* from, const uint32_t* to,
               const uint32_t* edge, const double* edge_w, DevCsr* out, cudaStream_t s) {
  out->n = n;
  out->arcs = arcs;
  out->off.alloc((size_t)n + 1);
  out->tgt.alloc(std::max<uint64_t>(arcs, 1));
  out->edge.alloc(std::max<uint64_t>(arcs, 1));
  if (edge_w) out->w.alloc(std::max<uint64_t>(arcs, 1));
  int tbits = bits_for(n);
  int fbits = bits_for(n);
  DevBuf<uint64_t> keys(std::max<uint64_t>(arcs, 1));
  DevBuf<uint32_t> vals(std::max<uint64_t>(arcs, 1));
  unsigned g = grid_for(arcs, 256);
  if (arcs) {
    make_keys<<<g, 256, 0, s>>>(from, to, edge, arcs, tbits, keys.get(), vals.get());
    KNB_LAUNCH("make_keys");
    radix_sort(keys.get(), vals.get(), arcs, tbits + fbits, s);
    split_keys<<<g, 256, 0, s>>>(keys.get(), vals.get(), arcs, tbits, edge_w, out->tgt.get(),
                                 out->edge.get(), edge_w ? out->w.get() : nullptr);
    KNB_LAUNCH("split_keys");
  }
  row_bounds<<<grid_for(arcs + 1, 256), 256, 0, s>>>(keys.get(), arcs, tbits, n, out->off.get());
  KNB_LAUNCH("row_bounds");
  KNB_CUDA(cudaStreamSynchronize(s));
}

__global__ void non_loop_flags(const uint32_t* __restrict__ src, const uint32_t* __restrict__ tgt,
                               uint64_t m, uint32_t* __restrict__ flag) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x)
    flag[e] = src[e] != tgt[e] ? 1u : 0u;
}

__global__ void expand_arcs(const uint32_t* __restrict__ src, const uint32_t* __restrict__ tgt,
                            uint64_t m, const uint32_t* __restrict__ before,
                            uint32_t* __restrict__ from, uint32_t* __restrict__ to,
                            uint32_t* __restrict__ edge) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t p = e + before[e];
    uint32_t a = src[e], b = tgt[e];
    from[p] = a;
    to[p] = b;
    edge[p] = (uint32_t)e;
    if (a != b) {
      from[p + 1] = b;
      to[p + 1] = a;
      edge[p + 1] = (uint32_t)e;
    }
  }
}

void build_undirected(uint32_t n, uint64_t m, const uint32_t* src, const uint32_t* tgt,
                      const double* w, DevCsr* out, cudaStream_t s) {
  DevBuf<uint32_t> flag(std::max<uint64_t>(m, 1));
  uint64_t nonloops = 0;
  if (m) {
    non_loop_flags<<<grid_for(m, 256), 256, 0, s>>>(src, tgt, m, flag.get());
    KNB_LAUNCH("non_loop_flags");
    nonloops = exclusive_scan<uint32_t>(flag.get(), flag.get(), m, s);
  }
  uint64_t arcs = m + nonloops;
  DevBuf<uint32_t> from(std::max<uint64_t>(arcs, 1)), to(std::max<uint64_t>(arcs, 1)),
      edge(std::max<uint64_t>(arcs, 1));
  if (m) {
    expand_arcs<<<grid_for(m, 256), 256, 0, s>>>(src, tgt, m, flag.get(), from.get(), to.get(),
                                                 edge.get());
    KNB_LAUNCH("expand_arcs");
  }
  build_csr(n, arcs, from.get(), to.get(), edge.get(), w, out, s);
}

const DevCsr& GraphHandleImpl::undirected_rows(cudaStream_t s) {
  if (!directed) return out;
  if (!und) {
    auto u = std::make_unique<DevCsr>();
    build_undirected(n, m, src.get(), tgt.get(), weighted ? w.get() : nullptr, u.get(), s);
    und = std::move(u);
  }
  return *und;
}

// ======================================================================= operators
// Arc values: weight (or 1) times the diagonal factor on self-loops
// (eigenvector.rs:512-547); FP32 copies and whether they are exact.
__global__ void op_values(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                          const double* __restrict__ w, uint32_t n, double lf,
                          double* __restrict__ v64, float* __restrict__ v32,
                          unsigned int* __restrict__ inexact) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    bool bad = false;
    for (uint32_t k = off[r]; k < off[r + 1]; ++k) {
      double x = w ? w[k] : 1.0;
      if (tgt[k] == r) x *= lf;
      v64[k] = x;
      float f = (float)x;
      v32[k] = f;
      if ((double)f != x) bad = true;
    }
    if (bad) atomicOr(inexact, 1u);
  }
}

__global__ void count_loops(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                            uint32_t n, unsigned long long* __restrict__ loops) {
  unsigned long long c = 0;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
    for (uint32_t k = off[r]; k < off[r + 1]; ++k) c += tgt[k] == r;
  c = warp_sum(c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(loops, c);
}

// Row sums in CSR order, one thread per row: for PageRank's pull operator
// the sums over the out-adjacency are the column sums of the in-adjacency
// operator in the reference's accumulation order (spectral.rs:240-246).
__global__ void row_sums_seq(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                             const double* __restrict__ w, uint32_t n, double lf,
                             double* __restrict__ sum, double* __restrict__ inv64,
                             float* __restrict__ inv32, unsigned int* __restrict__ dangling) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (uint32_t k = off[r]; k < off[r + 1]; ++k) {
      double x = w ? w[k] : 1.0;
      if (tgt[k] == r) x *= lf;
      s += x;
    }
    sum[r] = s;
    double inv = s > 0.0 ? 1.0 / s : 0.0;
    inv64[r] = inv;
    inv32[r] = (float)inv;
    if (!(s > 0.0)) atomicAdd(dangling, 1u);
  }
}

// Merge-path coordinates of tile boundaries (diagonal t * TILE).
__global__ void merge_coords(const uint32_t* __restrict__ off, uint32_t n, uint64_t nnz,
                             uint64_t tile, uint32_t ntiles, TileCoord* __restrict__ coords) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles;
       t += gridDim.x * blockDim.x) {
    uint64_t diag = std::min<uint64_t>((uint64_t)t * tile, (uint64_t)n + nnz);
    uint64_t lo = diag > nnz ? diag - nnz : 0, hi = std::min<uint64_t>(diag, n);
    while (lo < hi) {
      uint64_t mid = (lo + hi) >> 1;
      if ((uint64_t)off[mid + 1] <= diag - mid - 1) lo = mid + 1; else hi = mid;
    }
    coords[t].row = (uint32_t)lo;
    coords[t].arc = (uint32_t)(diag - lo);
  }
}

__global__ void gather_row_off(const TileCoord* __restrict__ coords, uint32_t ntiles,
                               const uint32_t* __restrict__ off, uint32_t n,
                               uint32_t* __restrict__ out) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t <= ntiles;
       t += gridDim.x * blockDim.x) {
    uint32_t r = coords[t].row;
    out[t] = r < n ? off[r] : 0xFFFFFFFFu;
  }
}

std::unique_ptr<Partition> build_partition(uint32_t n, uint64_t nnz, const uint32_t* off,
                                           uint32_t tile_items, cudaStream_t s) {
  auto p = std::make_unique<Partition>();
  p->tile = tile_items;
  uint64_t tile = tile_items;
  uint64_t items = (uint64_t)n + nnz;
  p->ntiles = (uint32_t)std::max<uint64_t>(1, (items + tile - 1) / tile);
  p->coords.alloc((size_t)p->ntiles + 1);
  merge_coords<<<grid_for(p->ntiles + 1, 256), 256, 0, s>>>(off, n, nnz, tile, p->ntiles,
                                                            p->coords.get());
  KNB_LAUNCH("merge_coords");
  DevBuf<uint32_t> roff((size_t)p->ntiles + 1);
  gather_row_off<<<grid_for(p->ntiles + 1, 256), 256, 0, s>>>(p->coords.get(), p->ntiles, off, n,
                                                              roff.get());
  KNB_LAUNCH("gather_row_off");
  std::vector<TileCoord> hc(p->ntiles + 1);
  std::vector<uint32_t> ho(p->ntiles + 1);
  KNB_CUDA(cudaMemcpyAsync(hc.data(), p->coords.get(), hc.size() * sizeof(TileCoord),
                           cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaMemcpyAsync(ho.data(), roff.get(), ho.size() * 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  // Rows open at the start of some tile cross a tile boundary; their first
  // tile holds their first arc, their last tile consumes their end marker.
  std::vector<SplitRow> sr;
  uint32_t T = p->ntiles;
  for (uint32_t t = 1; t < T; ++t) {
    uint32_t r = hc[t].row;
    if (r >= n || hc[t].arc <= ho[t]) continue;
    if (!sr.empty() && sr.back().row == r) continue;
    uint32_t first_arc = ho[t];
    // largest tile whose first arc index is <= first_arc
    uint32_t lo = 0, hi = t;  // answer in [0, t)
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) / 2;
      if (hc[mid].arc <= first_arc) lo = mid; else hi = mid;
    }
    uint32_t last = t;
    while (last + 1 < T && hc[last + 1].row == r) ++last;
    sr.push_back({r, lo, last});
  }
  std::stable_partition(sr.begin(), sr.end(),
                        [](const SplitRow& x) { return x.last - x.first <= SHORT_SPAN; });
  p->nshort = 0;
  while (p->nshort < sr.size() && sr[p->nshort].last - sr[p->nshort].first <= SHORT_SPAN)
    ++p->nshort;
  p->nsplit = (uint32_t)sr.size();
  p->split.alloc(std::max<size_t>(sr.size(), 1));
  if (!sr.empty())
    KNB_CUDA(cudaMemcpyAsync(p->split.get(), sr.data(), sr.size() * sizeof(SplitRow),
                             cudaMemcpyHostToDevice, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  return p;
}

const Partition& Operator::partition(uint32_t tile_items, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(mu);
  auto it = parts.find(tile_items);
  if (it != parts.end()) return *it->second;
  auto p = build_partition(n, nnz, rows->off.get(), tile_items, s);
  auto& ref = *p;
  parts[tile_items] = std::move(p);
  return ref;
}

// ----------------------------------------------------------------- relabelling
__global__ void relabel_keys(const uint32_t* __restrict__ toff, uint32_t n,
                             uint64_t* __restrict__ keys, uint32_t* __restrict__ ids) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    uint32_t cnt = toff[i + 1] - toff[i];
    keys[i] = ((uint64_t)(0xFFFFFFFFu - cnt) << 32) | i;
    ids[i] = i;
  }
}

__global__ void invert_perm(const uint32_t* __restrict__ perm, uint32_t n,
                            uint32_t* __restrict__ iperm) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    iperm[perm[k]] = k;
}

__global__ void permuted_lengths(const uint32_t* __restrict__ off, const uint32_t* __restrict__ perm,
                                 uint32_t n, uint32_t* __restrict__ len) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= n; k += gridDim.x * blockDim.x)
    len[k] = k < n ? off[perm[k] + 1] - off[perm[k]] : 0u;
}

// Arc q of the renumbered operator: its row by binary search over the new
// offsets, copied from the same position of the old row, column renamed.
__global__ void permuted_arcs(const uint32_t* __restrict__ off, const uint32_t* __restrict__ cols,
                              const double* __restrict__ v64, const float* __restrict__ v32,
                              const uint32_t* __restrict__ perm, const uint32_t* __restrict__ iperm,
                              const uint32_t* __restrict__ noff, uint32_t n, uint64_t nnz,
                              uint32_t* __restrict__ ncols, double* __restrict__ nv64,
                              float* __restrict__ nv32) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < nnz;
       q += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = n;  // largest k with noff[k] <= q
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) >> 1;
      if (noff[mid] <= q) lo = mid; else hi = mid;
    }
    uint64_t src = (uint64_t)off[perm[lo]] + (q - noff[lo]);
    ncols[q] = iperm[cols[src]];
    if (v64) {
      nv64[q] = v64[src];
      nv32[q] = v32[src];
    }
  }
}

template <class T>
__global__ void gather_vec(const T* __restrict__ in, const uint32_t* __restrict__ perm, uint32_t n,
                           T* __restrict__ out) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    out[k] = in[perm[k]];
}

const Relabeled& Operator::relabeled(cudaStream_t s) {
  std::lock_guard<std::mutex> lock(mu);
  if (relabel) return *relabel;
  auto r = std::make_unique<Relabeled>();
  const size_t nn = std::max<uint32_t>(n, 1);
  r->perm.alloc(nn);
  r->iperm.alloc(nn);
  r->off.alloc((size_t)n + 1);
  // arc arrays padded to the next multiple of 4 arcs, plus 4: the hot-node
  // sweep reads them with 16-byte loads from 16-byte boundaries
  const uint64_t arcs_padded = (nnz | 3) + 5;
  r->cols.alloc(arcs_padded);
  r->inv_out64.alloc(nn);
  r->inv_out32.alloc(nn);
  if (has_vals) {
    r->vals64.alloc(arcs_padded);
    r->vals32.alloc(arcs_padded);
  }
  {
    DevBuf<uint64_t> keys(nn);
    relabel_keys<<<grid_for(n, 256), 256, 0, s>>>(trans->off.get(), n, keys.get(), r->perm.get());
    KNB_LAUNCH("relabel_keys");
    radix_sort(keys.get(), r->perm.get(), n, 32 + bits_for(n), s);
  }
  invert_perm<<<grid_for(n, 256), 256, 0, s>>>(r->perm.get(), n, r->iperm.get());
  permuted_lengths<<<grid_for((uint64_t)n + 1, 256), 256, 0, s>>>(rows->off.get(), r->perm.get(), n,
                                                                  r->off.get());
  KNB_LAUNCH("relabel");
  exclusive_scan<uint32_t>(r->off.get(), r->off.get(), (size_t)n + 1, s);
  if (nnz) {
    permuted_arcs<<<grid_for(nnz, 256), 256, 0, s>>>(
        rows->off.get(), rows->tgt.get(), has_vals ? vals64.get() : nullptr,
        has_vals ? vals32.get() : nullptr, r->perm.get(), r->iperm.get(), r->off.get(), n, nnz,
        r->cols.get(), has_vals ? r->vals64.get() : nullptr, has_vals ? r->vals32.get() : nullptr);
    KNB_LAUNCH("permuted_arcs");
  }
  gather_vec<double><<<grid_for(n, 256), 256, 0, s>>>(inv_out64.get(), r->perm.get(), n,
                                                      r->inv_out64.get());
  gather_vec<float><<<grid_for(n, 256), 256, 0, s>>>(inv_out32.get(), r->perm.get(), n,
                                                     r->inv_out32.get());
  KNB_LAUNCH("gather_vec");
  KNB_CUDA(cudaStreamSynchronize(s));
  relabel = std::move(r);
  return *relabel;
}

const Partition& Operator::relabeled_partition(uint32_t tile_items, cudaStream_t s) {
  const Relabeled& r = relabeled(s);
  std::lock_guard<std::mutex> lock(mu);
  auto it = relabel->parts.find(tile_items);
  if (it != relabel->parts.end()) return *it->second;
  auto p = build_partition(n, nnz, r.off.get(), tile_items, s);
  auto& ref = *p;
  relabel->parts[tile_items] = std::move(p);
  return ref;
}

// ----------------------------------------------------------------- sliced layout
// Node order of the sliced layout: decreasing row length, then decreasing
// column count (how often a sweep gathers the node's value), then node.
__global__ void slice_node_keys(const uint32_t* __restrict__ off, const uint32_t* __restrict__ toff,
                                uint32_t n, uint64_t* __restrict__ keys, uint32_t* __restrict__ ids) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const uint32_t len = off[i + 1] - off[i];
    const uint32_t cnt = toff ? toff[i + 1] - toff[i] : 0u;
    keys[i] = ((uint64_t)(0xFFFFFFFFu - len) << 32) | (0xFFFFFFFFu - cnt);
    ids[i] = i;
  }
}

// Number of rows of at least lw arcs (lengths descend).
__global__ void slice_count_long(const uint32_t* __restrict__ len, uint32_t n, uint32_t lw,
                                 uint32_t* __restrict__ out) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    if (len[k] >= lw && (k + 1 == n || len[k + 1] < lw)) *out = k + 1;
}

// Arc a of the operator: key (new row, new column), payload a. The old row
// comes from a binary search over the old offsets.
__global__ void slice_arc_keys(const uint32_t* __restrict__ off, const uint32_t* __restrict__ cols,
                               const uint32_t* __restrict__ iperm, uint32_t n, uint64_t nnz,
                               int cbits, uint64_t* __restrict__ keys, uint32_t* __restrict__ ids) {
  for (uint64_t a = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; a < nnz;
       a += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = n;  // largest i with off[i] <= a
    while (hi - lo > 1) {
      const uint32_t mid = (lo + hi) >> 1;
      if (off[mid] <= a) lo = mid; else hi = mid;
    }
    keys[a] = ((uint64_t)iperm[lo] << cbits) | iperm[cols[a]];
    ids[a] = (uint32_t)a;
  }
}

// Elements of slice s: 32 times the length of its first row (the longest).
__global__ void slice_widths(const uint32_t* __restrict__ len, uint32_t n_long, uint32_t nslices,
                             uint64_t* __restrict__ w) {
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s <= nslices;
       s += gridDim.x * blockDim.x)
    w[s] = s < nslices ? 32ull * len[n_long + 32u * s] : 0ull;
}

// 32-bit slice bases and 16-bit lengths of the short rows.
__global__ void slice_small(const uint64_t* __restrict__ base64, const uint32_t* __restrict__ len,
                            uint32_t n_long, uint32_t n, uint32_t nslices,
                            uint32_t* __restrict__ base, uint16_t* __restrict__ slen) {
  const uint32_t count = max(n, nslices + 1);
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
    if (k <= nslices) base[k] = (uint32_t)base64[k];
    if (k >= n_long && k < n) slen[k - n_long] = (uint16_t)len[k];
  }
}

// Sorted arc q (key = new row << cbits | new column, payload = old arc):
// long rows go to the row-compressed part in order, short rows to element
// sbase[s] + 32 j + l of their slice (row n_long + 32 s + l, arc j).
__global__ void slice_place_arcs(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ ids,
                                 uint64_t nnz, int cbits, const uint32_t* __restrict__ noff,
                                 uint32_t n_long, uint32_t long_arcs,
                                 const uint32_t* __restrict__ sbase, const double* __restrict__ v64,
                                 const float* __restrict__ v32, uint32_t* __restrict__ lcols,
                                 double* __restrict__ lv64, float* __restrict__ lv32,
                                 uint32_t* __restrict__ scols, double* __restrict__ sv64,
                                 float* __restrict__ sv32) {
  const uint64_t cmask = (1ull << cbits) - 1;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < nnz;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t key = keys[q];
    const uint32_t col = (uint32_t)(key & cmask);
    const uint32_t a = ids[q];
    if (q < long_arcs) {
      lcols[q] = col;
      if (v64) {
        lv64[q] = v64[a];
        lv32[q] = v32[a];
      }
    } else {
      const uint32_t k = (uint32_t)(key >> cbits);
      const uint32_t j = (uint32_t)(q - noff[k]);
      const uint32_t rel = k - n_long;
      const uint64_t dst = (uint64_t)sbase[rel >> 5] + 32ull * j + (rel & 31u);
      scols[dst] = col;
      if (v64) {
        sv64[dst] = v64[a];
        sv32[dst] = v32[a];
      }
    }
  }
}

const SlicedOp& Operator::sliced(uint32_t lw, uint32_t pieces, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(lw, pieces);
  auto it = sliced_ops.find(key);
  if (it != sliced_ops.end()) return *it->second;
  if (lw < 1 || lw > 65535) throw Error("sliced layout: long-row threshold must be 1..65535");
  auto r = std::make_unique<SlicedOp>();
  r->n = n;
  r->nnz = nnz;
  r->lw = lw;
  r->has_vals = has_vals;
  const size_t nn = std::max<uint32_t>(n, 1);
  r->perm.alloc(nn);
  r->iperm.alloc(nn);
  r->inv_out64.alloc(nn);
  r->inv_out32.alloc(nn);
  {
    DevBuf<uint64_t> keys(nn);
    slice_node_keys<<<grid_for(n, 256), 256, 0, s>>>(rows->off.get(), trans ? trans->off.get() : nullptr,
                                                      n, keys.get(), r->perm.get());
    KNB_LAUNCH("slice_node_keys");
    radix_sort(keys.get(), r->perm.get(), n, 64, s);
  }
  invert_perm<<<grid_for(n, 256), 256, 0, s>>>(r->perm.get(), n, r->iperm.get());
  KNB_LAUNCH("invert_perm");
  DevBuf<uint32_t> nlen((size_t)n + 1), noff((size_t)n + 1);
  permuted_lengths<<<grid_for((uint64_t)n + 1, 256), 256, 0, s>>>(rows->off.get(), r->perm.get(), n,
                                                                  nlen.get());
  KNB_LAUNCH("permuted_lengths");
  const uint64_t total = exclusive_scan<uint32_t>(nlen.get(), noff.get(), (size_t)n + 1, s);
  if (total != nnz) throw Error("sliced layout: arc count mismatch");
  {
    DevBuf<uint32_t> cnt(1);
    KNB_CUDA(cudaMemsetAsync(cnt.get(), 0, 4, s));
    if (n) {
      slice_count_long<<<grid_for(n, 256), 256, 0, s>>>(nlen.get(), n, lw, cnt.get());
      KNB_LAUNCH("slice_count_long");
    }
    KNB_CUDA(cudaMemcpyAsync(&r->n_long, cnt.get(), 4, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
  }
  KNB_CUDA(cudaMemcpyAsync(&r->long_arcs, noff.get() + r->n_long, 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  r->nslices = (n - r->n_long + 31) / 32;
  // slice bases
  {
    DevBuf<uint64_t> w((size_t)r->nslices + 1);
    slice_widths<<<grid_for((uint64_t)r->nslices + 1, 256), 256, 0, s>>>(nlen.get(), r->n_long,
                                                                          r->nslices, w.get());
    KNB_LAUNCH("slice_widths");
    r->slice_elems = exclusive_scan<uint64_t>(w.get(), w.get(), (size_t)r->nslices + 1, s);
    if (r->slice_elems >= 0xFFFFFFFFull) throw Error("sliced layout: too many slice elements");
    r->sbase.alloc((size_t)r->nslices + 1);
    r->slen.alloc(std::max<size_t>((size_t)(n - r->n_long), 1));
    slice_small<<<grid_for(std::max<uint64_t>(n, (uint64_t)r->nslices + 1), 256), 256, 0, s>>>(
        w.get(), nlen.get(), r->n_long, n, r->nslices, r->sbase.get(), r->slen.get());
    KNB_LAUNCH("slice_small");
  }
  // arcs: sorted by (new row, new column), placed
  r->loff.alloc((size_t)r->n_long + 1);
  KNB_CUDA(cudaMemcpyAsync(r->loff.get(), noff.get(), ((size_t)r->n_long + 1) * 4,
                           cudaMemcpyDeviceToDevice, s));
  // long-row arrays end on a whole 32-arc block: bulk-staged sweeps copy
  // whole blocks (the tail past long_arcs is never added)
  const size_t long_alloc = ((size_t)r->long_arcs + 31) / 32 * 32 + 32;
  r->lcols.alloc(long_alloc);
  KNB_CUDA(cudaMemsetAsync(r->lcols.get() + r->long_arcs, 0, (long_alloc - r->long_arcs) * 4, s));
  r->scols.alloc(std::max<uint64_t>(r->slice_elems, 1));
  // slice padding (lanes shorter than their slice's first row) holds column
  // 0 and value 0; sweeps may load it but never gather or add it
  KNB_CUDA(cudaMemsetAsync(r->scols.get(), 0, r->scols.bytes(), s));
  if (has_vals) {
    r->lvals64.alloc(long_alloc);
    r->lvals32.alloc(long_alloc);
    KNB_CUDA(cudaMemsetAsync(r->lvals64.get() + r->long_arcs, 0,
                             (long_alloc - r->long_arcs) * sizeof(double), s));
    KNB_CUDA(cudaMemsetAsync(r->lvals32.get() + r->long_arcs, 0,
                             (long_alloc - r->long_arcs) * sizeof(float), s));
    r->svals64.alloc(std::max<uint64_t>(r->slice_elems, 1));
    r->svals32.alloc(std::max<uint64_t>(r->slice_elems, 1));
    KNB_CUDA(cudaMemsetAsync(r->svals64.get(), 0, r->svals64.bytes(), s));
    KNB_CUDA(cudaMemsetAsync(r->svals32.get(), 0, r->svals32.bytes(), s));
  }
  if (nnz) {
    const int cbits = std::max(1, bits_for(n));
    DevBuf<uint64_t> keys(nnz);
    DevBuf<uint32_t> ids(nnz);
    slice_arc_keys<<<grid_for(nnz, 256), 256, 0, s>>>(rows->off.get(), rows->tgt.get(),
                                                       r->iperm.get(), n, nnz, cbits, keys.get(),
                                                       ids.get());
    KNB_LAUNCH("slice_arc_keys");
    radix_sort(keys.get(), ids.get(), nnz, 2 * cbits, s);
    slice_place_arcs<<<grid_for(nnz, 256), 256, 0, s>>>(
        keys.get(), ids.get(), nnz, cbits, noff.get(), r->n_long, r->long_arcs, r->sbase.get(),
        has_vals ? vals64.get() : nullptr, has_vals ? vals32.get() : nullptr, r->lcols.get(),
        has_vals ? r->lvals64.get() : nullptr, has_vals ? r->lvals32.get() : nullptr,
        r->scols.get(), has_vals ? r->svals64.get() : nullptr,
        has_vals ? r->svals32.get() : nullptr);
    KNB_LAUNCH("slice_place_arcs");
  }
  gather_vec<double><<<grid_for(n, 256), 256, 0, s>>>(inv_out64.get(), r->perm.get(), n,
                                                      r->inv_out64.get());
  gather_vec<float><<<grid_for(n, 256), 256, 0, s>>>(inv_out32.get(), r->perm.get(), n,
                                                     r->inv_out32.get());
  KNB_LAUNCH("gather_vec");
  // pieces of the long rows, the row holding each piece's first arc, and the
  // rows a piece boundary cuts (their partials are added by split_rows)
  std::vector<uint32_t> hl((size_t)r->n_long + 1);
  KNB_CUDA(cudaMemcpyAsync(hl.data(), r->loff.get(), hl.size() * 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  const uint32_t want = std::max<uint32_t>(pieces, 1);
  uint32_t piece = r->long_arcs ? (uint32_t)(((uint64_t)r->long_arcs + want - 1) / want) : 1;
  piece = std::max<uint32_t>(32, (piece + 31) & ~31u);
  r->piece = piece;
  r->npieces = r->long_arcs ? (uint32_t)(((uint64_t)r->long_arcs + piece - 1) / piece) : 0;
  std::vector<uint32_t> prow(std::max<uint32_t>(r->npieces, 1), 0);
  {
    uint32_t row = 0;
    for (uint32_t t = 0; t < r->npieces; ++t) {
      const uint64_t a0 = (uint64_t)t * piece;
      while (row + 1 < r->n_long && hl[row + 1] <= a0) ++row;
      prow[t] = row;
    }
  }
  std::vector<SplitRow> sr;
  for (uint32_t row = 0; row < r->n_long; ++row) {
    const uint32_t first = hl[row] / piece, last = (hl[row + 1] - 1) / piece;
    if (first != last) sr.push_back({row, first, last});
  }
  std::stable_partition(sr.begin(), sr.end(),
                        [](const SplitRow& x) { return x.last - x.first <= SHORT_SPAN; });
  r->nshort = 0;
  while (r->nshort < sr.size() && sr[r->nshort].last - sr[r->nshort].first <= SHORT_SPAN)
    ++r->nshort;
  r->nsplit = (uint32_t)sr.size();
  r->prow.alloc(prow.size());
  KNB_CUDA(cudaMemcpyAsync(r->prow.get(), prow.data(), prow.size() * 4, cudaMemcpyHostToDevice, s));
  r->split.alloc(std::max<size_t>(sr.size(), 1));
  if (!sr.empty())
    KNB_CUDA(cudaMemcpyAsync(r->split.get(), sr.data(), sr.size() * sizeof(SplitRow),
                             cudaMemcpyHostToDevice, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  auto& ref = *r;
  sliced_ops[key] = std::move(r);
  return ref;
}

// Arc values from per-edge weights given by the caller (input edge order),
// through each arc's edge index.
__global__ void op_values_from_edges(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                                     const uint32_t* __restrict__ edge, const double* __restrict__ w,
                                     uint32_t n, double lf, double* __restrict__ v64,
                                     float* __restrict__ v32, unsigned int* __restrict__ inexact) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    bool bad = false;
    for (uint32_t k = off[r]; k < off[r + 1]; ++k) {
      double x = w[edge[k]];
      if (tgt[k] == r) x *= lf;
      v64[k] = x;
      float f = (float)x;
      v32[k] = f;
      if ((double)f != x) bad = true;
    }
    if (bad) atomicOr(inexact, 1u);
  }
}

__global__ void row_sums_from_edges(const uint32_t* __restrict__ off, const uint32_t* __restrict__ tgt,
                                    const uint32_t* __restrict__ edge, const double* __restrict__ w,
                                    uint32_t n, double lf, double* __restrict__ sum,
                                    double* __restrict__ inv64, float* __restrict__ inv32,
                                    unsigned int* __restrict__ dangling) {
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (uint32_t k = off[r]; k < off[r + 1]; ++k) {
      double x = w[edge[k]];
      if (tgt[k] == r) x *= lf;
      s += x;
    }
    sum[r] = s;
    double inv = s > 0.0 ? 1.0 / s : 0.0;
    inv64[r] = inv;
    inv32[r] = (float)inv;
    if (!(s > 0.0)) atomicAdd(dangling, 1u);
  }
}

// An operator over the chosen rows with value buffers allocated (not filled).
static std::unique_ptr<Operator> weights_skeleton(GraphHandleImpl& g, int which, cudaStream_t s) {
  auto o = std::make_unique<Operator>();
  const DevCsr* rows = which == 0 ? &g.out : which == 1 ? &g.in_rows() : &g.undirected_rows(s);
  const DevCsr* trans = which == 0 ? &g.in_rows() : which == 1 ? &g.out : rows;
  o->rows = rows;
  o->trans = trans;
  o->n = g.n;
  o->nnz = rows->arcs;
  o->has_vals = true;
  o->vals64.alloc(std::max<uint64_t>(o->nnz, 1));
  o->vals32.alloc(std::max<uint64_t>(o->nnz, 1));
  o->colsum.alloc(std::max<uint32_t>(g.n, 1));
  o->inv_out64.alloc(std::max<uint32_t>(g.n, 1));
  o->inv_out32.alloc(std::max<uint32_t>(g.n, 1));
  return o;
}

void GraphHandleImpl::fill_weights(Operator& o, const double* d_w, double lf, cudaStream_t s) {
  const DevCsr* rows = o.rows;
  const DevCsr* trans = o.trans;
  DevBuf<unsigned int> flags(2);
  KNB_CUDA(cudaMemsetAsync(flags.get(), 0, 8, s));
  if (n) {
    op_values_from_edges<<<grid_for(n, 256), 256, 0, s>>>(rows->off.get(), rows->tgt.get(),
                                                          rows->edge.get(), d_w, n, lf,
                                                          o.vals64.get(), o.vals32.get(),
                                                          flags.get());
    row_sums_from_edges<<<grid_for(n, 128), 128, 0, s>>>(trans->off.get(), trans->tgt.get(),
                                                         trans->edge.get(), d_w, n, lf,
                                                         o.colsum.get(), o.inv_out64.get(),
                                                         o.inv_out32.get(), flags.get() + 1);
    KNB_LAUNCH("weighted_op");
  }
  unsigned int hf[2] = {0, 0};
  KNB_CUDA(cudaMemcpyAsync(hf, flags.get(), 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  o.vals32_exact = hf[0] == 0;
  o.n_dangling = hf[1];
}

GraphHandleImpl::WeightSlot& GraphHandleImpl::weight_slot(int which, double lf, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_pair(which, (int)(lf * 2));
  auto& slot = wslots[key];
  if (!slot) {
    slot = std::make_unique<WeightSlot>();
    slot->op = weights_skeleton(*this, which, s);
  }
  return *slot;
}

Operator& GraphHandleImpl::op(int which, bool wtd, double lf, cudaStream_t s) {
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_tuple(which, wtd ? 1 : 0, (int)(lf * 2));
  auto it = ops.find(key);
  if (it != ops.end()) return *it->second;
  auto o = std::make_unique<Operator>();
  const DevCsr* rows = which == 0 ? &out : which == 1 ? &in_rows() : &undirected_rows(s);
  // The transpose whose row sums are this operator's column sums.
  const DevCsr* trans = which == 0 ? &in_rows() : which == 1 ? &out : rows;
  o->rows = rows;
  o->trans = trans;
  o->n = n;
  o->nnz = rows->arcs;
  const double* wv = (wtd && weighted) ? rows->w.get() : nullptr;
  const double* wt = (wtd && weighted) ? trans->w.get() : nullptr;
  DevBuf<unsigned long long> loops(1);
  KNB_CUDA(cudaMemsetAsync(loops.get(), 0, 8, s));
  if (n) {
    count_loops<<<grid_for(n, 256), 256, 0, s>>>(rows->off.get(), rows->tgt.get(), n, loops.get());
    KNB_LAUNCH("count_loops");
  }
  unsigned long long nloops = 0;
  KNB_CUDA(cudaMemcpyAsync(&nloops, loops.get(), 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  o->has_vals = wv != nullptr || (lf != 1.0 && nloops > 0);
  DevBuf<unsigned int> flags(2);
  KNB_CUDA(cudaMemsetAsync(flags.get(), 0, 8, s));
  if (o->has_vals && o->nnz) {
    o->vals64.alloc(o->nnz);
    o->vals32.alloc(o->nnz);
    op_values<<<grid_for(n, 256), 256, 0, s>>>(rows->off.get(), rows->tgt.get(), wv, n, lf,
                                               o->vals64.get(), o->vals32.get(), flags.get());
    KNB_LAUNCH("op_values");
  }
  o->colsum.alloc(std::max<uint32_t>(n, 1));
  o->inv_out64.alloc(std::max<uint32_t>(n, 1));
  o->inv_out32.alloc(std::max<uint32_t>(n, 1));
  if (n) {
    row_sums_seq<<<grid_for(n, 128), 128, 0, s>>>(trans->off.get(), trans->tgt.get(), wt, n, lf,
                                                  o->colsum.get(), o->inv_out64.get(),
                                                  o->inv_out32.get(), flags.get() + 1);
    KNB_LAUNCH("row_sums_seq");
  }
  unsigned int hf[2] = {0, 0};
  KNB_CUDA(cudaMemcpyAsync(hf, flags.get(), 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  o->vals32_exact = hf[0] == 0;
  o->n_dangling = hf[1];
  auto& ref = *o;
  ops[key] = std::move(o);
  return ref;
}

}  // namespace knb
