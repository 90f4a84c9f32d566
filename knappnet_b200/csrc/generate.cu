// Synthetic inputs on the device: R-MAT edges (Chakrabarti, Zhan and
// Faloutsos 2004) and lognormal arc strengths, both from Philox4x32-10
// counter-based streams (Salmon et al. 2011) named (seed, index) as in the
// reference's rng.rs, so the same seed gives the same graph on any device
// and on the CPU.
#include "generate.cuh"

namespace knb {

__device__ __forceinline__ void philox_block(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                             uint32_t k0, uint32_t k1, uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

// Edge k: `scale` words of stream (seed, k), most significant level first.
__global__ void rmat_edges(int scale, uint64_t m, uint32_t ta, uint32_t tab, uint32_t tabc,
                           uint64_t seed, uint32_t* __restrict__ src, uint32_t* __restrict__ tgt) {
  const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < m;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t r = 0, q = 0;
    uint32_t w[4];
    for (int l = 0; l < scale; ++l) {
      if ((l & 3) == 0) {
        uint64_t blk = (uint64_t)(l >> 2);
        philox_block((uint32_t)blk, (uint32_t)(blk >> 32), (uint32_t)k, (uint32_t)(k >> 32), k0, k1, w);
      }
      uint32_t u = w[l & 3];
      uint32_t rb = u >= tab ? 1u : 0u;
      uint32_t cb = ((u >= ta && u < tab) || u >= tabc) ? 1u : 0u;
      r = r << 1 | rb;
      q = q << 1 | cb;
    }
    src[k] = r;
    tgt[k] = q;
  }
}

// Keys for cleaning: loops flagged out; (min, max) when symmetrizing.
__global__ void rmat_keys(const uint32_t* __restrict__ src, const uint32_t* __restrict__ tgt,
                          uint64_t m, int scale, int symmetrize, uint64_t* __restrict__ keys,
                          uint32_t* __restrict__ keep) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < m;
       k += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a = src[k], b = tgt[k];
    if (symmetrize && a > b) {
      uint32_t t = a;
      a = b;
      b = t;
    }
    keys[k] = ((uint64_t)a << scale) | b;
    keep[k] = a != b;
  }
}

__global__ void compact_keys(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ keep,
                             const uint32_t* __restrict__ pos, uint64_t m,
                             uint64_t* __restrict__ out) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < m;
       k += (uint64_t)gridDim.x * blockDim.x)
    if (keep[k]) out[pos[k]] = keys[k];
}

__global__ void first_of_run(const uint64_t* __restrict__ keys, uint64_t m,
                             uint32_t* __restrict__ flag) {
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < m;
       k += (uint64_t)gridDim.x * blockDim.x)
    flag[k] = (k == 0 || keys[k] != keys[k - 1]) ? 1u : 0u;
}

__global__ void unique_split(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ flag,
                             const uint32_t* __restrict__ pos, uint64_t m, int scale,
                             uint32_t* __restrict__ src, uint32_t* __restrict__ tgt) {
  const uint64_t mask = (1ull << scale) - 1;
  for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < m;
       k += (uint64_t)gridDim.x * blockDim.x)
    if (flag[k]) {
      src[pos[k]] = (uint32_t)(keys[k] >> scale);
      tgt[pos[k]] = (uint32_t)(keys[k] & mask);
    }
}

// w_e = exp(z), z = sqrt(-2 ln(1 - u1)) cos(2 pi u2) (Box and Muller 1958),
// u1, u2 the first two 53-bit uniforms of stream (wseed, e); rounded to FP32.
__global__ void lognormal_weights(uint64_t m, uint64_t wseed, float* __restrict__ w) {
  const uint32_t k0 = (uint32_t)wseed, k1 = (uint32_t)(wseed >> 32);
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t r[4];
    philox_block(0, 0, (uint32_t)e, (uint32_t)(e >> 32), k0, k1, r);
    uint64_t a = ((uint64_t)r[0] << 32) | r[1], b = ((uint64_t)r[2] << 32) | r[3];
    double u1 = (double)(a >> 11) * (1.0 / 9007199254740992.0);
    double u2 = (double)(b >> 11) * (1.0 / 9007199254740992.0);
    double z = sqrt(-2.0 * log(1.0 - u1)) * cos(6.283185307179586 * u2);
    w[e] = (float)exp(z);
  }
}

RmatEdges generate_rmat(int scale, uint64_t edge_factor, double a, double b, double c,
                        uint64_t seed, bool clean, bool symmetrize, bool lognormal, uint64_t wseed,
                        cudaStream_t s) {
  if (scale < 1 || scale > 31) throw Error("R-MAT scale must be between 1 and 31");
  if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0))
    throw Error("R-MAT probabilities must be nonnegative with a + b + c <= 1");
  const uint64_t m = edge_factor << scale;
  if (m > 0xFFFFFFFFull / 2) throw Error("R-MAT edge count exceeds the supported maximum");
  const double two32 = 4294967296.0;
  auto th = [&](double p) -> uint32_t {
    double t = p * two32;
    return t >= two32 ? 0xFFFFFFFFu : (uint32_t)t;
  };
  RmatEdges out;
  out.n = 1u << scale;
  DevBuf<uint32_t> src(m), tgt(m);
  rmat_edges<<<grid_for(m, 256, 148 * 64), 256, 0, s>>>(scale, m, th(a), th(a + b), th(a + b + c),
                                                        seed, src.get(), tgt.get());
  KNB_LAUNCH("rmat_edges");
  if (!clean && !symmetrize) {
    out.m = m;
    out.src = std::move(src);
    out.tgt = std::move(tgt);
  } else {
    DevBuf<uint64_t> keys(m);
    DevBuf<uint32_t> keep(m + 1);
    rmat_keys<<<grid_for(m, 256), 256, 0, s>>>(src.get(), tgt.get(), m, scale, symmetrize ? 1 : 0,
                                               keys.get(), keep.get());
    KNB_LAUNCH("rmat_keys");
    DevBuf<uint32_t> pos(m + 1);
    uint64_t kept = exclusive_scan<uint32_t>(keep.get(), pos.get(), m, s);
    DevBuf<uint64_t> ck(std::max<uint64_t>(kept, 1));
    compact_keys<<<grid_for(m, 256), 256, 0, s>>>(keys.get(), keep.get(), pos.get(), m, ck.get());
    KNB_LAUNCH("compact_keys");
    keys.release();
    src.release();
    tgt.release();
    DevBuf<uint32_t> dummy(std::max<uint64_t>(kept, 1));
    KNB_CUDA(cudaMemsetAsync(dummy.get(), 0, std::max<uint64_t>(kept, 1) * 4, s));
    radix_sort(ck.get(), dummy.get(), kept, 2 * scale, s);
    DevBuf<uint32_t> flag(std::max<uint64_t>(kept, 1)), fpos(std::max<uint64_t>(kept, 1));
    uint64_t uniq = 0;
    if (kept) {
      first_of_run<<<grid_for(kept, 256), 256, 0, s>>>(ck.get(), kept, flag.get());
      uniq = exclusive_scan<uint32_t>(flag.get(), fpos.get(), kept, s);
    }
    out.m = uniq;
    out.src.alloc(std::max<uint64_t>(uniq, 1));
    out.tgt.alloc(std::max<uint64_t>(uniq, 1));
    if (kept) {
      unique_split<<<grid_for(kept, 256), 256, 0, s>>>(ck.get(), flag.get(), fpos.get(), kept,
                                                       scale, out.src.get(), out.tgt.get());
      KNB_LAUNCH("unique_split");
    }
  }
  if (lognormal) {
    out.w32.alloc(std::max<uint64_t>(out.m, 1));
    if (out.m) {
      lognormal_weights<<<grid_for(out.m, 256), 256, 0, s>>>(out.m, wseed, out.w32.get());
      KNB_LAUNCH("lognormal_weights");
    }
  }
  KNB_CUDA(cudaStreamSynchronize(s));
  return out;
}

}  // namespace knb

// ======================================================================= G(n, m)
// Host generator of G(n, m) graphs with the reference's algorithm
// (crates/engine/src/generate.rs:255-290): Floyd's sampling of m distinct
// candidate pairs from stream (seed, rep), decoded and sorted.
#include <algorithm>
#include <cmath>
#include <thread>
#include <unordered_set>

namespace knb {
namespace {

struct HostStream {
  uint32_t k0, k1;
  uint64_t stream, block = 0;
  uint32_t buf[4];
  int used = 4;
  HostStream(uint64_t seed, uint64_t index)
      : k0((uint32_t)seed), k1((uint32_t)(seed >> 32)), stream(index) {}
  uint32_t next_u32() {
    if (used == 4) {
      uint32_t c0 = (uint32_t)block, c1 = (uint32_t)(block >> 32), c2 = (uint32_t)stream,
               c3 = (uint32_t)(stream >> 32), a = k0, b = k1;
      for (int r = 0; r < 10; ++r) {
        if (r) {
          a += 0x9E3779B9u;
          b += 0xBB67AE85u;
        }
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ a, n2 = (uint32_t)(p0 >> 32) ^ c3 ^ b;
        c0 = n0;
        c1 = (uint32_t)p1;
        c2 = n2;
        c3 = (uint32_t)p0;
      }
      buf[0] = c0;
      buf[1] = c1;
      buf[2] = c2;
      buf[3] = c3;
      ++block;
      used = 0;
    }
    return buf[used++];
  }
  uint64_t next_u64() {
    uint64_t hi = next_u32();
    return hi << 32 | next_u32();
  }
  uint64_t below(uint64_t n) {
    const uint64_t mx = ~0ull;
    const uint64_t zone = mx - (mx % n + 1) % n;
    for (;;) {
      uint64_t x = next_u64();
      if (x <= zone) return x % n;
    }
  }
  double uniform() { return (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0); }
};

uint64_t pair_count(uint64_t n, bool directed, bool loops) {
  if (directed) return loops ? n * n : n * (n ? n - 1 : 0);
  return loops ? n * (n + 1) / 2 : n * (n ? n - 1 : 0) / 2;
}

uint64_t isqrt(uint64_t x) {
  uint64_t r = (uint64_t)std::sqrt((double)x);
  while (r > 0 && r * r > x) --r;
  while ((r + 1) * (r + 1) <= x) ++r;
  return r;
}

void decode(uint64_t k, uint64_t n, bool directed, bool loops, uint64_t* a, uint64_t* b) {
  if (directed && loops) {
    *a = k / n;
    *b = k % n;
  } else if (directed) {
    uint64_t row = k / (n - 1), col = k % (n - 1);
    *a = row;
    *b = col >= row ? col + 1 : col;
  } else if (!loops) {
    uint64_t c = (1 + isqrt(1 + 8 * k)) / 2;
    while (c * (c - 1) / 2 > k) --c;
    while ((c + 1) * c / 2 <= k) ++c;
    *a = k - c * (c - 1) / 2;
    *b = c;
  } else {
    uint64_t c = (isqrt(1 + 8 * k) - 1) / 2;
    while (c * (c + 1) / 2 > k) --c;
    while ((c + 1) * (c + 2) / 2 <= k) ++c;
    *a = k - c * (c + 1) / 2;
    *b = c;
  }
}

}  // namespace

void gnm_edges(uint64_t n, uint64_t m, bool directed, bool loops, uint64_t seed, uint64_t rep,
               int64_t offset, int64_t* src, int64_t* tgt) {
  HostStream rng(seed, rep);
  const uint64_t total = pair_count(n, directed, loops);
  if (m > total) throw Error("a graph on " + std::to_string(n) + " nodes cannot hold " +
                             std::to_string(m) + " edges");
  std::vector<uint64_t> chosen;
  chosen.reserve(m);
  if (m * 2 <= total) {
    std::unordered_set<uint64_t> set;
    set.reserve(m * 2);
    for (uint64_t j = total - m; j < total; ++j) {
      uint64_t t = rng.below(j + 1);
      if (!set.insert(t).second) set.insert(j);
    }
    chosen.assign(set.begin(), set.end());
  } else {
    std::unordered_set<uint64_t> skip;
    for (uint64_t j = m; j < total; ++j) {
      uint64_t t = rng.below(j + 1);
      if (!skip.insert(t).second) skip.insert(j);
    }
    for (uint64_t k = 0; k < total; ++k)
      if (!skip.count(k)) chosen.push_back(k);
  }
  std::vector<std::pair<uint64_t, uint64_t>> pairs(chosen.size());
  for (size_t i = 0; i < chosen.size(); ++i) decode(chosen[i], n, directed, loops, &pairs[i].first, &pairs[i].second);
  std::sort(pairs.begin(), pairs.end());
  for (size_t i = 0; i < pairs.size(); ++i) {
    src[i] = (int64_t)pairs[i].first + offset;
    tgt[i] = (int64_t)pairs[i].second + offset;
  }
}

// Graph k of a batch uses stream (seed, k) and node offset sum(n[0..k)).
void gnm_batch(uint64_t count, const int64_t* n, const int64_t* m, bool directed, bool loops,
               uint64_t seed, int64_t* src, int64_t* tgt, int threads) {
  std::vector<int64_t> noff(count + 1, 0), eoff(count + 1, 0);
  for (uint64_t k = 0; k < count; ++k) {
    noff[k + 1] = noff[k] + n[k];
    eoff[k + 1] = eoff[k] + m[k];
  }
  if (threads <= 0) threads = (int)std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::thread> pool;
  std::vector<std::string> errors(threads);
  for (int t = 0; t < threads; ++t) {
    pool.emplace_back([&, t] {
      try {
        for (uint64_t k = t; k < count; k += threads)
          gnm_edges((uint64_t)n[k], (uint64_t)m[k], directed, loops, seed, k, noff[k],
                    src + eoff[k], tgt + eoff[k]);
      } catch (const std::exception& e) {
        errors[t] = e.what();
      }
    });
  }
  for (auto& th : pool) th.join();
  for (auto& e : errors)
    if (!e.empty()) throw Error(e);
}

// Sizes from a power law p(x) ~ x^-alpha on [lo, hi] by inverse transform of
// the continuous law, floored; size k from stream (seed, k).
void power_law_sizes(uint64_t count, double alpha, double lo, double hi, uint64_t seed,
                     int64_t* out) {
  const double e = 1.0 - alpha;
  const double a = std::pow(lo, e), b = std::pow(hi, e);
  for (uint64_t k = 0; k < count; ++k) {
    HostStream rng(seed, k);
    const double u = rng.uniform();
    double x = std::pow(a + u * (b - a), 1.0 / e);
    int64_t v = (int64_t)std::floor(x);
    out[k] = std::min<int64_t>(std::max<int64_t>(v, (int64_t)lo), (int64_t)hi);
  }
}

}  // namespace knb
