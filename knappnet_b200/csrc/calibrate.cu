// Gather-rate calibration: random 4-byte loads per second that the whole GPU
// sustains from a device array (L2-resident when it fits), from each SM's own
// shared memory, and from the shared memory of a thread-block cluster. The
// sparse sweeps gather their iterate at random, so the first figure bounds
// how fast any sweep can gather what L1 does not hold; the other two show
// what a shared-memory or cluster-distributed cache of the iterate could
// give. Every kernel here only reads its own buffers with hashed indices;
// the cluster kernel's only waits are the two cluster barriers every CTA of
// the cluster executes.
#include <cooperative_groups.h>

#include <string>

#include "calibrate.cuh"

namespace cg = cooperative_groups;

namespace knb {

namespace {

constexpr int CAL_THREADS = 1024;
constexpr int CAL_ITERS = 256;
constexpr uint32_t CAL_SMEM_WORDS = 49152;  // 192 KB of FP32 per CTA

__device__ __forceinline__ uint32_t cal_hash(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352dU;
  x ^= x >> 15;
  x *= 0x846ca68bU;
  x ^= x >> 16;
  return x;
}

__global__ void __launch_bounds__(CAL_THREADS) cal_array_gather(const float* __restrict__ x,
                                                                uint32_t n, float* __restrict__ sink) {
  uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  float s = 0.f;
#pragma unroll 8
  for (int i = 0; i < CAL_ITERS; ++i) {
    h = cal_hash(h + (uint32_t)i);
    s += __ldcg(x + h % n);
  }
  if (s == 1234.5f) sink[0] = s;  // never true for the zero-filled array; keeps the loads
}

__global__ void __launch_bounds__(CAL_THREADS) cal_smem_gather(const float* __restrict__ x,
                                                               float* __restrict__ sink) {
  extern __shared__ float cal_sm[];
  for (uint32_t i = threadIdx.x; i < CAL_SMEM_WORDS; i += blockDim.x) cal_sm[i] = x[i];
  __syncthreads();
  uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  float s = 0.f;
#pragma unroll 8
  for (int i = 0; i < CAL_ITERS; ++i) {
    h = cal_hash(h + (uint32_t)i);
    s += cal_sm[h % CAL_SMEM_WORDS];
  }
  if (s == 1234.5f) sink[0] = s;
}

template <int C>
__global__ void __launch_bounds__(CAL_THREADS) cal_cluster_gather(const float* __restrict__ x,
                                                                  float* __restrict__ sink) {
  extern __shared__ float cal_sm[];
  cg::cluster_group cl = cg::this_cluster();
  for (uint32_t i = threadIdx.x; i < CAL_SMEM_WORDS; i += blockDim.x) cal_sm[i] = x[i];
  cl.sync();  // every CTA's copy is in place before any is read
  float* part[C];
#pragma unroll
  for (int r = 0; r < C; ++r) part[r] = cl.map_shared_rank(cal_sm, r);
  uint32_t h = blockIdx.x * blockDim.x + threadIdx.x;
  float s = 0.f;
#pragma unroll 8
  for (int i = 0; i < CAL_ITERS; ++i) {
    h = cal_hash(h + (uint32_t)i);
    s += part[(h >> 24) % C][h % CAL_SMEM_WORDS];
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
  if (s == 1234.5f) sink[0] = s;
}

// Times `launch` (a few waves of CTAs) five times after two untimed runs.
template <class F>
double timed_rate(F launch, double gathers_per_launch, cudaStream_t s) {
  for (int w = 0; w < 2; ++w) launch();
  cudaEvent_t a, b;
  KNB_CUDA(cudaEventCreate(&a));
  KNB_CUDA(cudaEventCreate(&b));
  KNB_CUDA(cudaEventRecord(a, s));
  for (int r = 0; r < 5; ++r) launch();
  KNB_CUDA(cudaEventRecord(b, s));
  KNB_CUDA(cudaEventSynchronize(b));
  float ms = 0.f;
  KNB_CUDA(cudaEventElapsedTime(&ms, a, b));
  KNB_CUDA(cudaEventDestroy(a));
  KNB_CUDA(cudaEventDestroy(b));
  return gathers_per_launch * 5.0 / ((double)ms * 1e-3);
}

template <int C>
double cluster_rate(const float* x, float* sink, cudaStream_t s) {
  auto fn = cal_cluster_gather<C>;
  const size_t smem = (size_t)CAL_SMEM_WORDS * 4;
  KNB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(CAL_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  KNB_CUDA(cudaOccupancyMaxActiveClusters(&clusters, (const void*)fn, &cfg));
  if (clusters < 1) throw Error("no cluster of " + std::to_string(C) + " CTAs fits");
  cfg.gridDim = dim3((unsigned)(clusters * C * 4));
  const double per_launch = (double)clusters * C * 4 * CAL_THREADS * CAL_ITERS;
  return timed_rate([&] { KNB_CUDA(cudaLaunchKernelEx(&cfg, fn, x, sink)); }, per_launch, s);
}

}  // namespace

double measure_gather_rate(int source, uint64_t words, cudaStream_t s) {
  if (source != 0 && source != 1 && source != 2 && source != 4 && source != 8)
    throw Error("gather source must be 0 (device array), 1 (shared memory) or 2, 4, 8 (cluster)");
  if (source == 0 && (words < 1024 || words > (1ull << 31)))
    throw Error("the array must hold between 1024 and 2^31 values");
  const uint64_t n = source == 0 ? words : CAL_SMEM_WORDS;
  DevBuf<float> x(n), sink(1);
  KNB_CUDA(cudaMemsetAsync(x.get(), 0, n * 4, s));
  int dev = 0, sms = 0;
  KNB_CUDA(cudaGetDevice(&dev));
  KNB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (source == 0) {
    const unsigned grid = (unsigned)sms * 2 * 4;
    const double per_launch = (double)grid * CAL_THREADS * CAL_ITERS;
    return timed_rate([&] {
      cal_array_gather<<<grid, CAL_THREADS, 0, s>>>(x.get(), (uint32_t)n, sink.get());
      KNB_LAUNCH("cal_array_gather");
    }, per_launch, s);
  }
  if (source == 1) {
    const size_t smem = (size_t)CAL_SMEM_WORDS * 4;
    KNB_CUDA(cudaFuncSetAttribute(cal_smem_gather, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem));
    const unsigned grid = (unsigned)sms * 4;
    const double per_launch = (double)grid * CAL_THREADS * CAL_ITERS;
    return timed_rate([&] {
      cal_smem_gather<<<grid, CAL_THREADS, smem, s>>>(x.get(), sink.get());
      KNB_LAUNCH("cal_smem_gather");
    }, per_launch, s);
  }
  if (source == 2) return cluster_rate<2>(x.get(), sink.get(), s);
  if (source == 4) return cluster_rate<4>(x.get(), sink.get(), s);
  return cluster_rate<8>(x.get(), sink.get(), s);
}

}  // namespace knb
