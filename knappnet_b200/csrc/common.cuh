// Shared device and host helpers of the knappnet B200 library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>

namespace knb {

// ---------------------------------------------------------------- errors
// Every failure below the C ABI is a C++ exception carrying the message the
// ABI writes into the caller's err buffer.
struct Error : std::runtime_error {
  explicit Error(const std::string& m) : std::runtime_error(m) {}
};

inline void cuda_check(cudaError_t e, const char* what) {
  if (e != cudaSuccess)
    throw Error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
}
#define KNB_CUDA(x) ::knb::cuda_check((x), #x)
#define KNB_LAUNCH(what) ::knb::cuda_check(cudaGetLastError(), what)

constexpr int WARP = 32;

// ---------------------------------------------------------------- L2 cache policy
// Streamed arrays (column indices, arc values) are read once per sweep and
// should not push the gathered iterate out of the 126 MB L2; the iterate
// should stay. createpolicy builds the 64-bit L2 cache-policy operands.
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// Read-only loads with an L2 policy (ld.global.nc.L2::cache_hint). They are
// not `volatile`, so the compiler may batch independent loads ahead of their
// uses (a volatile asm would keep every gather in program order).
__device__ __forceinline__ uint32_t ld_stream(const uint32_t* p, uint64_t pol) {
  uint32_t v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.u32 %0, [%1], %2;"
               : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_stream(const float* p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;"
               : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_stream(const double* p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;"
               : "=d"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_keep(const float* p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_keep(const double* p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}

// 16-byte streamed loads (four u32 / f32, or two f64); the address must be
// 16-byte aligned.
__device__ __forceinline__ void ld_stream4(const uint32_t* p, uint64_t pol, uint32_t (&o)[4]) {
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0, %1, %2, %3}, [%4], %5;"
      : "=r"(o[0]), "=r"(o[1]), "=r"(o[2]), "=r"(o[3]) : "l"(p), "l"(pol));
}
__device__ __forceinline__ void ld_stream4(const float* p, uint64_t pol, float (&o)[4]) {
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
      : "=f"(o[0]), "=f"(o[1]), "=f"(o[2]), "=f"(o[3]) : "l"(p), "l"(pol));
}
__device__ __forceinline__ void ld_stream4(const double* p, uint64_t pol, double (&o)[4]) {
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
      : "=d"(o[0]), "=d"(o[1]) : "l"(p), "l"(pol));
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
      : "=d"(o[2]), "=d"(o[3]) : "l"(p + 2), "l"(pol));
}

// Gathers that skip L1 allocation (the L2 policy still applies).
__device__ __forceinline__ float ld_keep_na(const float* p, uint64_t pol) {
  float v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_keep_na(const double* p, uint64_t pol) {
  double v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(p), "l"(pol));
  return v;
}

// ---------------------------------------------------------------- reductions
template <class T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
// Sums of K <= 4 per-lane values over a warp by a reduce-scatter butterfly:
// the first two exchanges also halve the number of values a lane carries,
// so the K sums cost 2 + 1 + 3 shuffles instead of 5 K. Returns, in every
// lane, the warp sum of value lane / 8 (lanes 8 K and up return a sum of
// zeros). The association is fixed, so results are identical run to run.
template <int K>
__device__ __forceinline__ double warp_sum_scatter(const double* v, int lane) {
  static_assert(K >= 1 && K <= 4, "at most 4 values");
  constexpr unsigned F = 0xffffffffu;
  const double v0 = v[0], v1 = K > 1 ? v[1] : 0.0, v2 = K > 2 ? v[2] : 0.0,
               v3 = K > 3 ? v[3] : 0.0;
  const bool h16 = (lane & 16) != 0, h8 = (lane & 8) != 0;
  // lanes 0-15 keep values 0 and 1, lanes 16-31 values 2 and 3
  const double a0 = __shfl_xor_sync(F, h16 ? v0 : v2, 16);
  const double a1 = __shfl_xor_sync(F, h16 ? v1 : v3, 16);
  const double k0 = (h16 ? v2 : v0) + a0;
  const double k1 = (h16 ? v3 : v1) + a1;
  // then lanes with bit 3 clear keep the even value of the pair, set the odd
  const double b = __shfl_xor_sync(F, h8 ? k0 : k1, 8);
  double m = (h8 ? k1 : k0) + b;
  m += __shfl_xor_sync(F, m, 4);
  m += __shfl_xor_sync(F, m, 2);
  m += __shfl_xor_sync(F, m, 1);
  return m;
}

// Epilogues whose per-tile scalars are all plain sums declare SUMS = true.
template <class E, class = void>
struct EpiSums {
  static constexpr bool value = false;
};
template <class E>
struct EpiSums<E, std::void_t<decltype(E::SUMS)>> {
  static constexpr bool value = E::SUMS;
};

template <class T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum in a fixed order (warp butterflies, then warp 0 over the
// warp totals), so the result is the same on every run. `scratch` holds at
// least blockDim.x / 32 values. The total is returned to every thread.
template <class T>
__device__ __forceinline__ T block_sum(T v, T* scratch) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[w] = v;
  __syncthreads();
  T t = lane < nw ? scratch[lane] : T(0);
  t = warp_sum(t);
  return t;
}
template <class T>
__device__ __forceinline__ T block_max(T v, T* scratch) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) scratch[w] = v;
  __syncthreads();
  T t = lane < nw ? scratch[lane] : T(-1e308);
  t = warp_max(t);
  return t;
}

// ---------------------------------------------------------------- launch helpers
// Sets a kernel attribute on the current device unless this process already
// set it to the same value there: cudaFuncSetAttribute acts on the current
// device only, and graph handles may live on any device, so the record is
// kept per (kernel, device, attribute), under a lock shared by all threads.
inline void set_func_attr(const void* fn, cudaFuncAttribute attr, int value) {
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, int>, int> applied;
  int dev = 0;
  cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_tuple(fn, dev, (int)attr);
  auto it = applied.find(key);
  if (it != applied.end() && it->second == value) return;
  cuda_check(cudaFuncSetAttribute(fn, attr, value), "cudaFuncSetAttribute");
  applied[key] = value;
}

inline unsigned grid_for(uint64_t work, unsigned block, unsigned cap = 148u * 32u) {
  uint64_t g = (work + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

// Device memory owned by RAII (freed with cudaFree on destruction).
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t count) { alloc(count); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      p = o.p; n = o.n; o.p = nullptr; o.n = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t count) {
    release();
    n = count;
    if (count) {
      cudaError_t e = cudaMalloc(&p, count * sizeof(T));
      if (e != cudaSuccess) {
        p = nullptr;
        n = 0;
        throw Error("out of device memory allocating " + std::to_string(count * sizeof(T)) +
                    " bytes");
      }
    }
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  T* get() const { return p; }
  size_t bytes() const { return n * sizeof(T); }
};

}  // namespace knb
