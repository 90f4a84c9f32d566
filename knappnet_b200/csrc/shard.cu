// Row shards of one graph's PageRank (see shard.cuh for the split sweep).
// Reference loop: crates/engine/src/metrics/spectral.rs:247-280.
#include <algorithm>

#include "shard.cuh"

namespace knb {
namespace {

constexpr int SH_THREADS = 256;
constexpr unsigned SH_GRID_CAP = 1184;  // 8 CTAs of 256 per SM
constexpr int SH_MAX_PARTS = 1024;
constexpr uint32_t SH_UNROLL = 4;  // elements a thread loads at once in shard_finish

// One thread per boundary: the first row r with r + off[r] >= k (n + nnz) /
// parts (r + off[r] grows strictly with r, and is n + nnz at r = n).
__global__ void shard_bounds_kernel(const uint32_t* __restrict__ off, uint32_t n, uint64_t nnz,
                                    int parts, int64_t* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k > parts) return;
  const uint64_t target = ((uint64_t)n + nnz) * (uint64_t)k / (uint64_t)parts;
  uint32_t lo = 0, hi = n;  // the answer lies in [lo, hi]
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if ((uint64_t)mid + off[mid] >= target) hi = mid; else lo = mid + 1;
  }
  out[k] = lo;
}

// The shard's row offsets, from 0.
__global__ void shard_rebase(const uint32_t* __restrict__ off, uint32_t r0, uint32_t rows,
                             uint32_t* __restrict__ out) {
  const uint32_t base = off[r0];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= rows;
       i += gridDim.x * blockDim.x)
    out[i] = off[r0 + i] - base;
}

// dst[i] = src[perm[base + i]] for i < count.
__global__ void shard_gather(const double* __restrict__ src, const uint32_t* __restrict__ perm,
                             uint32_t base, uint32_t count, double* __restrict__ dst) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count;
       i += gridDim.x * blockDim.x)
    dst[i] = src[perm[base + i]];
}

// dst[perm[k]] = src[k] for k < n (back to node order).
__global__ void shard_scatter(const double* __restrict__ src, const uint32_t* __restrict__ perm,
                              uint32_t n, double* __restrict__ dst) {
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
    dst[perm[k]] = src[k];
}

__device__ __forceinline__ bool shard_last(unsigned int* ticket) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (last) __threadfence();
  return last;
}

// Sum of slot s of K-wide partials of nb CTAs, in a fixed order.
template <int K>
__device__ __forceinline__ double shard_parts(const double* part, uint32_t nb, int s,
                                              double* scratch) {
  const volatile double* p = part;
  double a = 0;
  for (uint32_t q = threadIdx.x; q < nb; q += blockDim.x) a += p[(size_t)q * K + s];
  return block_sum(a, scratch);
}

// y_i = d (y_i + D jump_i) + (1 - d) p_i over the shard's rows (y_i is the
// product A z on entry), the padding zeroed, and the fixed-order sum of the
// rows' values in the payload's last slot.
__global__ void __launch_bounds__(SH_THREADS)
shard_update(double* __restrict__ y, uint32_t rows, size_t payload_len, double d,
             const double* __restrict__ p, bool jump_uniform, double inv_n,
             double* __restrict__ part, ShardState* st) {
  __shared__ double sh[SH_THREADS / 32];
  const double stuck = st->stuck;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  double t = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < rows; i += stride) {
    const double pi = p ? p[i] : inv_n;
    const double ji = jump_uniform ? inv_n : pi;
    const double v = d * (y[i] + stuck * ji) + (1.0 - d) * pi;
    y[i] = v;
    t += v;
  }
  for (size_t i = rows + (size_t)blockIdx.x * blockDim.x + threadIdx.x; i + 1 < payload_len;
       i += stride)
    y[i] = 0.0;
  t = block_sum(t, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
  if (!shard_last(&st->ticket)) return;
  const double total = shard_parts<1>(part, gridDim.x, 0, sh);
  if (threadIdx.x == 0) {
    y[payload_len - 1] = total;
    st->ticket = 0;
  }
}

// Over all n nodes: x' = y / T from the gathered payloads (or 1/n to start,
// g null), change = sum |x' - x|, z = x' / out (0 where out is 0) and the
// dangling mass D = sum of x' over those nodes.
__global__ void __launch_bounds__(SH_THREADS)
shard_finish_kernel(const double* __restrict__ g, size_t L, const int64_t* __restrict__ bounds,
                    int parts, uint32_t n, double* __restrict__ x, double* __restrict__ z,
                    const double* __restrict__ out, double inv_n, double* __restrict__ part,
                    ShardState* st) {
  __shared__ double sh[SH_THREADS / 32];
  __shared__ int64_t sb[SH_MAX_PARTS + 1];
  __shared__ double total;
  for (int k = threadIdx.x; k <= parts; k += blockDim.x) sb[k] = bounds[k];
  if (threadIdx.x == 0 && g) {
    double t = 0;
    for (int k = 0; k < parts; ++k) t += g[(size_t)k * L + L - 1];
    total = t;
  }
  __syncthreads();
  // A thread visits i = t, t + stride, ... in that order, SH_UNROLL at a
  // time: all their loads first, so that the divisions (whose rare slow path
  // is a branch) do not hold each load back behind the previous one.
  const uint32_t stride = gridDim.x * blockDim.x;
  double ch = 0, dg = 0;
  for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += SH_UNROLL * stride) {
    double gv[SH_UNROLL], xv[SH_UNROLL], ov[SH_UNROLL];
#pragma unroll
    for (int u = 0; u < SH_UNROLL; ++u) {
      const uint32_t i = i0 + u * stride;
      gv[u] = inv_n;
      xv[u] = 0.0;
      ov[u] = 0.0;
      if (i < n) {
        if (g) {
          // the last rank whose range starts at or before i owns it
          // (ranges are contiguous and may be empty)
          int lo = 0, hi = parts - 1;
          while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (sb[mid] <= (int64_t)i) lo = mid; else hi = mid - 1;
          }
          gv[u] = g[(size_t)lo * L + (size_t)((int64_t)i - sb[lo])];
          xv[u] = x[i];
        }
        ov[u] = out[i];
      }
    }
#pragma unroll
    for (int u = 0; u < SH_UNROLL; ++u) {
      const uint32_t i = i0 + u * stride;
      if (i >= n) break;
      double xn = inv_n;
      if (g) {
        xn = gv[u] / total;
        ch += fabs(xn - xv[u]);
      }
      x[i] = xn;
      if (ov[u] > 0.0) {
        z[i] = xn / ov[u];
      } else {
        z[i] = 0.0;
        dg += xn;
      }
    }
  }
  ch = block_sum(ch, sh);
  dg = block_sum(dg, sh);
  if (threadIdx.x == 0) {
    part[blockIdx.x * 2] = ch;
    part[blockIdx.x * 2 + 1] = dg;
  }
  if (!shard_last(&st->ticket)) return;
  const double c = shard_parts<2>(part, gridDim.x, 0, sh);
  const double dm = shard_parts<2>(part, gridDim.x, 1, sh);
  if (threadIdx.x == 0) {
    st->change = c;
    st->stuck = dm;
    st->ticket = 0;
  }
}

void launch_finish(Shard& sh, const double* g, cudaStream_t s) {
  const unsigned gv = grid_for(sh.n, SH_THREADS, SH_GRID_CAP);
  shard_finish_kernel<<<gv, SH_THREADS, 0, s>>>(g, sh.payload_len, sh.dbounds.get(), sh.parts,
                                               sh.n, sh.x.get(), sh.z.get(), sh.out.get(),
                                               1.0 / (double)sh.n, sh.part_all.get(),
                                               sh.st.get());
  KNB_LAUNCH("shard_finish");
}

}  // namespace

Shard::~Shard() {
  if (hst) cudaFreeHost(hst);
}

std::vector<int64_t> shard_bounds(Operator& op, int parts, cudaStream_t s) {
  if (parts < 1 || parts > SH_MAX_PARTS)
    throw Error("the number of shards must be between 1 and " + std::to_string(SH_MAX_PARTS));
  std::vector<int64_t> h((size_t)parts + 1, 0);
  if (op.n == 0) return h;
  const Relabeled& R = op.relabeled(s);
  DevBuf<int64_t> d((size_t)parts + 1);
  shard_bounds_kernel<<<grid_for((uint64_t)parts + 1, 256), 256, 0, s>>>(
      R.off.get(), op.n, op.nnz, parts, d.get());
  KNB_LAUNCH("shard_bounds");
  KNB_CUDA(cudaMemcpyAsync(h.data(), d.get(), h.size() * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  return h;
}

std::unique_ptr<Shard> shard_new(Operator& op, double damping, const double* d_pers,
                                 bool jump_uniform, const std::vector<int64_t>& bounds,
                                 int rank, cudaStream_t s) {
  const int parts = (int)bounds.size() - 1;
  if (parts < 1 || parts > SH_MAX_PARTS)
    throw Error("the number of shards must be between 1 and " + std::to_string(SH_MAX_PARTS));
  if (rank < 0 || rank >= parts)
    throw Error("shard " + std::to_string(rank) + " is outside [0, " + std::to_string(parts) +
                ")");
  if (bounds[0] != 0 || bounds[parts] != (int64_t)op.n)
    throw Error("shard bounds must start at 0 and end at the node count " +
                std::to_string(op.n));
  size_t widest = 0;
  for (int k = 0; k < parts; ++k) {
    if (bounds[k + 1] < bounds[k]) throw Error("shard bounds must not decrease");
    widest = std::max<size_t>(widest, (size_t)(bounds[k + 1] - bounds[k]));
  }
  auto sh = std::make_unique<Shard>();
  sh->op = &op;
  sh->n = op.n;
  sh->parts = parts;
  sh->rank = rank;
  sh->r0 = (uint32_t)bounds[rank];
  sh->r1 = (uint32_t)bounds[rank + 1];
  sh->bounds = bounds;
  sh->damping = damping;
  sh->pers = d_pers != nullptr;
  sh->jump_uniform = jump_uniform;
  // the widest range, then the partial sum, rounded up to 32 doubles
  sh->payload_len = (widest + 1 + 31) / 32 * 32;
  const uint32_t rows = sh->r1 - sh->r0;
  sh->dbounds.alloc((size_t)parts + 1);
  KNB_CUDA(cudaMemcpyAsync(sh->dbounds.get(), bounds.data(), bounds.size() * 8,
                           cudaMemcpyHostToDevice, s));
  sh->off.alloc((size_t)rows + 1);
  uint32_t o[2] = {0, 0};
  sh->x.alloc(std::max<uint32_t>(sh->n, 1));
  sh->z.alloc(std::max<uint32_t>(sh->n, 1));
  sh->out.alloc(std::max<uint32_t>(sh->n, 1));
  if (sh->n > 0) {
    sh->rl = &op.relabeled(s);
    const uint32_t* roff = sh->rl->off.get();
    shard_rebase<<<grid_for((uint64_t)rows + 1, 256), 256, 0, s>>>(roff, sh->r0, rows,
                                                                 sh->off.get());
    KNB_LAUNCH("shard_rebase");
    shard_gather<<<grid_for(sh->n, 256), 256, 0, s>>>(op.colsum.get(), sh->rl->perm.get(), 0,
                                                      sh->n, sh->out.get());
    KNB_LAUNCH("shard_gather");
    KNB_CUDA(cudaMemcpyAsync(&o[0], roff + sh->r0, 4, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaMemcpyAsync(&o[1], roff + sh->r1, 4, cudaMemcpyDeviceToHost, s));
  }
  KNB_CUDA(cudaStreamSynchronize(s));
  sh->arc0 = o[0];
  sh->arcs = (uint64_t)(o[1] - o[0]);
  if (rows > 0) sh->part = build_partition(rows, sh->arcs, sh->off.get(), product_tile(), s);
  if (d_pers) {
    sh->p.alloc(std::max<uint32_t>(rows, 1));
    if (rows > 0) {
      shard_gather<<<grid_for(rows, 256), 256, 0, s>>>(d_pers, sh->rl->perm.get(), sh->r0, rows,
                                                       sh->p.get());
      KNB_LAUNCH("shard_gather");
    }
  }
  sh->part_rows.alloc((size_t)grid_for(std::max<uint32_t>(rows, 1), SH_THREADS, SH_GRID_CAP) + 8);
  sh->part_all.alloc((size_t)grid_for(std::max<uint32_t>(sh->n, 1), SH_THREADS, SH_GRID_CAP) * 2 +
                     8);
  sh->st.alloc(1);
  KNB_CUDA(cudaMemsetAsync(sh->st.get(), 0, sizeof(ShardState), s));
  KNB_CUDA(cudaMallocHost(&sh->hst, sizeof(ShardState)));
  if (sh->n > 0) launch_finish(*sh, nullptr, s);
  KNB_CUDA(cudaStreamSynchronize(s));
  return sh;
}

void shard_sweep(Shard& sh, double* d_payload, cudaStream_t s) {
  const uint32_t rows = sh.r1 - sh.r0;
  if (rows > 0) {
    const Operator& op = *sh.op;
    const OpView<double> v{rows, sh.arcs, sh.off.get(), sh.rl->cols.get() + sh.arc0,
                           op.has_vals ? sh.rl->vals64.get() + sh.arc0 : nullptr};
    product64(v, *sh.part, sh.z.get(), d_payload, sh.scratch, s);
  }
  const unsigned gr = grid_for(std::max<uint32_t>(rows, 1), SH_THREADS, SH_GRID_CAP);
  shard_update<<<gr, SH_THREADS, 0, s>>>(d_payload, rows, sh.payload_len, sh.damping,
                                         sh.pers ? sh.p.get() : nullptr, sh.jump_uniform,
                                         1.0 / (double)std::max<uint32_t>(sh.n, 1),
                                         sh.part_rows.get(), sh.st.get());
  KNB_LAUNCH("shard_update");
}

void shard_scores(Shard& sh, double* out, bool out_on_device, cudaStream_t s) {
  if (sh.n == 0) return;
  double* dst = out;
  if (!out_on_device) {
    if (!sh.scores.p) sh.scores.alloc(sh.n);
    dst = sh.scores.get();
  }
  shard_scatter<<<grid_for(sh.n, 256), 256, 0, s>>>(sh.x.get(), sh.rl->perm.get(), sh.n, dst);
  KNB_LAUNCH("shard_scatter");
  if (!out_on_device)
    KNB_CUDA(cudaMemcpyAsync(out, dst, (size_t)sh.n * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
}

void shard_restart(Shard& sh, cudaStream_t s) {
  if (sh.n > 0) launch_finish(sh, nullptr, s);
}

double shard_finish(Shard& sh, const double* d_gathered, cudaStream_t s) {
  if (sh.n == 0) return 0.0;
  launch_finish(sh, d_gathered, s);
  KNB_CUDA(cudaMemcpyAsync(sh.hst, sh.st.get(), sizeof(ShardState), cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  return sh.hst->change;
}

}  // namespace knb
