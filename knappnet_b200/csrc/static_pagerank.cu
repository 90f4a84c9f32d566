// PageRank of one graph given as device arrays, without allocating device
// memory.
//
// Some callers cannot call cudaMalloc: hosts whose framework has reserved
// the device memory for its own allocator (so a stray cudaMalloc fails or
// fragments that pool), and code paths that must not stall the device
// (cudaMalloc and cudaFree may synchronize it). For them this file offers one
// entry point, net_pagerank_csr_static, whose scratch memory (iterates,
// out-strengths, a status word) lives in a file-scope __device__ array of
// fixed size, sized for graphs of up to KNB_STATIC_MAX_NODES nodes. Every GPU
// that loads the library holds that array until the process exits.
//
// The kernel is the single-graph form of the packed-graph PageRank
// (ego.cu): one CTA runs the reference's iteration
// (crates/engine/src/metrics/spectral.rs:247-280) with CTA-wide reductions
// in a fixed order, so repeated calls give identical results.
//
// The array's address is looked up with cudaGetSymbolAddress once per device,
// on the first call made with that device current; that first call should
// therefore come before any stream capture. All calls share the one array,
// and the kernel resets what must start at zero, so calls run one after
// another are independent; calls that overlap on the GPU (concurrent streams
// or threads on one device) race on the array and must be serialized by the
// caller.
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/knappnet.h"
#include "common.cuh"

namespace {

// Largest graph the static scratch holds: 2^18 nodes (four FP64 vectors of
// that length, 8 MiB).
constexpr uint32_t KNB_STATIC_MAX_NODES = 1u << 18;
constexpr int STATIC_THREADS = 1024;
constexpr int STATIC_LOG_THREADS = 10;
constexpr unsigned long long NONE = ULLONG_MAX;

// Status words written by every launch: [0] iterations, [1] converged,
// [2] first row whose offsets decrease, [3] first arc whose source is not a
// node, [4] that source, [5] first arc whose weight is negative or not
// finite, [6] that weight's bits. Entries 2, 3 and 5 hold -1 when no arc or
// row is at fault.
constexpr int NSTATUS = 7;

static __device__ __align__(256) double g_static_scratch[4 * KNB_STATIC_MAX_NODES];
static __device__ __align__(256) int64_t g_static_status[NSTATUS];

__device__ __forceinline__ double cta_sum_static(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = knb::warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  for (int k = 0; k < nw; ++k) t += sh[k];
  return t;
}

// Ascending bitonic sort of the CTA's STATIC_THREADS keys in shared memory.
__device__ __forceinline__ void cta_sort_keys(unsigned long long* key) {
  const uint32_t t = threadIdx.x;
  for (uint32_t k = 2; k <= (uint32_t)STATIC_THREADS; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      const uint32_t p = t ^ j;
      if (p > t) {
        const unsigned long long a = key[t], b = key[p];
        const bool up = (t & k) == 0;
        if ((a > b) == up) {
          key[t] = b;
          key[p] = a;
        }
      }
      __syncthreads();
    }
  }
}

// scratch: [x | y | z | out-strength], each KNB_STATIC_MAX_NODES long.
__global__ void __launch_bounds__(STATIC_THREADS)
static_pagerank(uint32_t n, const uint32_t* __restrict__ off, const uint32_t* __restrict__ src,
                const double* __restrict__ w, double d, double tol, int64_t max_iter,
                double* __restrict__ scratch, int64_t* __restrict__ status,
                double* __restrict__ out) {
  __shared__ double sh[32];
  __shared__ unsigned long long skey[STATIC_THREADS];
  __shared__ double sw[STATIC_THREADS];
  __shared__ unsigned long long bad_off, bad_src, bad_w;
  double* x = scratch;
  double* y = scratch + KNB_STATIC_MAX_NODES;
  double* z = scratch + 2 * (size_t)KNB_STATIC_MAX_NODES;
  double* os = scratch + 3 * (size_t)KNB_STATIC_MAX_NODES;
  const uint32_t tid = threadIdx.x;
  if (tid == 0) bad_off = bad_src = bad_w = NONE;
  // out-strength: column sums of the in-arc rows (reset first: the array
  // keeps the previous call's contents)
  for (uint32_t i = tid; i < n; i += blockDim.x) os[i] = 0.0;
  __syncthreads();
  for (uint32_t i = tid; i < n; i += blockDim.x)
    if (off[i + 1] < off[i]) atomicMin(&bad_off, (unsigned long long)i);
  __syncthreads();
  if (bad_off == NONE) {
    // The arcs, STATIC_THREADS at a time in arc order. Each chunk is sorted
    // by (source, position in the chunk) and the first arc of every run of
    // one source adds the run's weights in arc order, then adds that to the
    // source's out-strength: one writer per source per chunk and chunks in
    // order, so every column sum has a fixed association.
    const uint32_t a0 = off[0], a1 = off[n];
    for (uint64_t base = a0; base < a1; base += STATIC_THREADS) {
      const uint64_t k = base + tid;
      unsigned long long key = NONE;
      double wv = 0.0;
      if (k < a1) {
        const uint32_t s = src[k];
        wv = w ? w[k] : 1.0;
        if (s >= n) atomicMin(&bad_src, (unsigned long long)k);
        else if (!(wv >= 0.0) || isinf(wv)) atomicMin(&bad_w, (unsigned long long)k);
        else key = ((unsigned long long)s << STATIC_LOG_THREADS) | tid;
      }
      skey[tid] = key;
      sw[tid] = wv;
      __syncthreads();
      cta_sort_keys(skey);
      const unsigned long long kk = skey[tid];
      if (kk != NONE) {
        const unsigned long long s = kk >> STATIC_LOG_THREADS;
        if (tid == 0 || (skey[tid - 1] >> STATIC_LOG_THREADS) != s) {
          double acc = 0.0;
          for (uint32_t q = tid; q < (uint32_t)STATIC_THREADS && skey[q] != NONE &&
                                 (skey[q] >> STATIC_LOG_THREADS) == s;
               ++q)
            acc += sw[skey[q] & (STATIC_THREADS - 1)];
          os[s] += acc;
        }
      }
      __syncthreads();
    }
  }
  if (bad_off != NONE || bad_src != NONE || bad_w != NONE) {
    // nothing below runs on arrays that failed a check
    if (tid == 0) {
      status[0] = 0;
      status[1] = 0;
      status[2] = bad_off == NONE ? -1 : (int64_t)bad_off;
      status[3] = bad_src == NONE ? -1 : (int64_t)bad_src;
      status[4] = bad_src == NONE ? 0 : (int64_t)src[bad_src];
      status[5] = bad_w == NONE ? -1 : (int64_t)bad_w;
      status[6] = bad_w == NONE ? 0 : __double_as_longlong(w[bad_w]);
    }
    return;
  }
  const double inv_n = 1.0 / (double)n;
  for (uint32_t i = tid; i < n; i += blockDim.x) x[i] = inv_n;
  __syncthreads();
  int64_t it = 0;
  int converged = 0;
  while (it < max_iter) {
    double stuck = 0;
    for (uint32_t i = tid; i < n; i += blockDim.x) {
      const double o = os[i];
      if (o > 0.0) {
        z[i] = x[i] / o;
      } else {
        z[i] = 0.0;
        stuck += x[i];
      }
    }
    stuck = cta_sum_static(stuck, sh);
    double total = 0;
    for (uint32_t i = tid; i < n; i += blockDim.x) {
      double s = 0;
      for (uint32_t k = off[i]; k < off[i + 1]; ++k) s += (w ? w[k] : 1.0) * z[src[k]];
      const double v = d * (s + stuck * inv_n) + (1.0 - d) * inv_n;
      y[i] = v;
      total += v;
    }
    total = cta_sum_static(total, sh);
    double change = 0;
    for (uint32_t i = tid; i < n; i += blockDim.x) {
      const double v = y[i] / total;
      y[i] = v;
      change += fabs(v - x[i]);
    }
    change = cta_sum_static(change, sh);
    double* t = x;
    x = y;
    y = t;
    ++it;
    if (change <= tol) {
      converged = 1;
      break;
    }
  }
  for (uint32_t i = tid; i < n; i += blockDim.x) out[i] = x[i];
  if (tid == 0) {
    status[0] = it;
    status[1] = converged;
    status[2] = status[3] = status[5] = -1;
    status[4] = status[6] = 0;
  }
}

struct StaticSymbols {
  double* scratch = nullptr;
  int64_t* status = nullptr;
};

// Device addresses of the static arrays, looked up once per device with
// that device current.
bool static_symbols(int dev, StaticSymbols* out, std::string* why) {
  static std::mutex mu;
  static StaticSymbols table[64];
  static bool ready[64] = {false};
  if (dev < 0 || dev >= 64) {
    *why = "device ordinal out of range";
    return false;
  }
  std::lock_guard<std::mutex> lock(mu);
  if (!ready[dev]) {
    StaticSymbols s;
    cudaError_t e1 = cudaGetSymbolAddress((void**)&s.scratch, g_static_scratch);
    if (e1 != cudaSuccess) {
      *why = std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e1);
      return false;
    }
    cudaError_t e2 = cudaGetSymbolAddress((void**)&s.status, g_static_status);
    if (e2 != cudaSuccess) {
      *why = std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e2);
      return false;
    }
    table[dev] = s;
    ready[dev] = true;
  }
  *out = table[dev];
  return true;
}

void write_static_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  size_t k = msg.size() < len - 1 ? msg.size() : len - 1;
  memcpy(err, msg.data(), k);
  err[k] = 0;
}

std::string fmt_static(double v) {
  char b[64];
  snprintf(b, sizeof b, "%g", v);
  return b;
}

}  // namespace

extern "C" int32_t net_pagerank_csr_static(int64_t n, const uint32_t* d_offsets,
                                           const uint32_t* d_sources, const double* d_weights,
                                           double damping, double tol, int64_t max_iter,
                                           double* d_out, int64_t* iterations, void* stream,
                                           char* err, size_t err_len) {
  if (n < 0) {
    write_static_err(err, err_len, "negative node count");
    return 1;
  }
  if ((uint64_t)n > KNB_STATIC_MAX_NODES) {
    write_static_err(err, err_len,
                     "the graph has " + std::to_string(n) +
                         " nodes; net_pagerank_csr_static holds at most " +
                         std::to_string(KNB_STATIC_MAX_NODES) +
                         " nodes in its static scratch memory (use net_pagerank)");
    return 1;
  }
  if (!(damping >= 0.0 && damping <= 1.0)) {
    write_static_err(err, err_len,
                     "damping is " + fmt_static(damping) + "; it must be between 0 and 1");
    return 1;
  }
  if (n == 0) {
    if (iterations) *iterations = 0;
    return 0;
  }
  if (!d_offsets || !d_sources || !d_out) {
    write_static_err(err, err_len, "a device array is null");
    return 1;
  }
  // A tolerance that is not positive (NaN included) and a cap that is not
  // positive select the defaults, as net_pagerank does.
  const double t = tol > 0 ? tol : 1e-12;
  const int64_t cap = max_iter > 0 ? max_iter : 10000;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    write_static_err(err, err_len, std::string("CUDA error: ") + cudaGetErrorString(e));
    return 1;
  }
  StaticSymbols sym;
  std::string why;
  if (!static_symbols(dev, &sym, &why)) {
    write_static_err(err, err_len, why);
    return 1;
  }
  cudaStream_t s = (cudaStream_t)stream;
  static_pagerank<<<1, STATIC_THREADS, 0, s>>>((uint32_t)n, d_offsets, d_sources, d_weights, damping,
                                               t, cap, sym.scratch, sym.status, d_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    write_static_err(err, err_len, std::string("CUDA error: ") + cudaGetErrorString(e));
    return 1;
  }
  int64_t st[NSTATUS] = {0};
  e = cudaMemcpyAsync(st, sym.status, sizeof st, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    write_static_err(err, err_len, std::string("CUDA error: ") + cudaGetErrorString(e));
    return 1;
  }
  if (st[2] >= 0) {
    write_static_err(err, err_len, "the row offsets decrease after row " + std::to_string(st[2]));
    return 1;
  }
  if (st[3] >= 0) {
    write_static_err(err, err_len, "arc " + std::to_string(st[3]) + " has source " +
                                       std::to_string(st[4]) + ", outside the graph's " +
                                       std::to_string(n) + " nodes");
    return 1;
  }
  if (st[5] >= 0) {
    double wv = 0;
    memcpy(&wv, &st[6], sizeof wv);
    write_static_err(err, err_len,
                     std::isfinite(wv)
                         ? "arc " + std::to_string(st[5]) + " has negative weight " +
                               fmt_static(wv) + "; PageRank requires non-negative weights"
                         : "arc " + std::to_string(st[5]) + " has weight " + fmt_static(wv) +
                               "; PageRank requires finite, non-negative weights");
    return 1;
  }
  if (iterations) *iterations = st[0];
  if (!st[1]) {
    write_static_err(err, err_len, "PageRank did not converge to tolerance " + fmt_static(t) +
                                       " within " + std::to_string(cap) + " iterations");
    return 1;
  }
  return 0;
}
