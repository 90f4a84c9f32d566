// The C ABI of the B200 library: the reference's netcapi.h entry points for
// the spectral-centrality path, with its argument meaning, defaults and error
// behaviour (crates/capi/src/lib.rs:57-212, crates/capi/src/spectral.rs:35-97,
// crates/capi/src/topography.rs:208-249), plus additive extensions declared
// in include/knappnet.h.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <limits>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/knappnet.h"
#include "adjoint.cuh"
#include "batch.cuh"
#include "ego.cuh"
#include "eigen.cuh"
#include "frame.cuh"
#include "calibrate.cuh"
#include "katz.cuh"
#include "generate.cuh"
#include "graph.cuh"
#include "pagerank.cuh"
#include "shard.cuh"

using knb::Error;

struct GraphHandle {
  knb::GraphHandleImpl g;
};

struct NetShard {
  std::unique_ptr<knb::Shard> s;
};

namespace {

void write_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  size_t k = std::min(msg.size(), len - 1);
  memcpy(err, msg.data(), k);
  err[k] = 0;
}

template <class F>
int32_t guard(char* err, size_t len, F f) {
  try {
    f();
    return 0;
  } catch (const Error& e) {
    write_err(err, len, e.what());
  } catch (const std::bad_alloc&) {
    write_err(err, len, "out of host memory in the network engine");
  } catch (const std::exception& e) {
    write_err(err, len, std::string("internal error in the network engine: ") + e.what());
  } catch (...) {
    write_err(err, len, "internal error in the network engine");
  }
  return 1;
}

knb::GraphHandleImpl& handle(const GraphHandle* h) {
  if (!h) throw Error("graph handle is null");
  return const_cast<GraphHandle*>(h)->g;
}

std::string fmt_g(double v) {
  char b[64];
  snprintf(b, sizeof b, "%g", v);
  return b;
}

// The tolerance a call runs with: the given value when it is positive, else
// the default 1e-12. NaN is not positive, so it also selects the default,
// as in the reference's wrappers (crates/capi/src/spectral.rs:36-42,
// crates/capi/src/topography.rs:232).
double tolerance(double tol) { return tol > 0 ? tol : 1e-12; }

// ---------------------------------------------------------------- device checks
// First invalid endpoint, as 2 * edge + (0 for source, 1 for target), so the
// smallest value names the edge and endpoint the reference reports first
// (crates/engine/src/graph.rs:182-194).
__global__ void convert_edges(const int64_t* __restrict__ s64, const int64_t* __restrict__ t64,
                              uint64_t m, uint64_t n, uint32_t* __restrict__ s32,
                              uint32_t* __restrict__ t32, unsigned long long* __restrict__ bad) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    int64_t a = s64[e], b = t64[e];
    bool ba = a < 0 || (uint64_t)a >= n, bb = b < 0 || (uint64_t)b >= n;
    if (ba) atomicMin(bad, (unsigned long long)(2 * e));
    else if (bb) atomicMin(bad, (unsigned long long)(2 * e + 1));
    s32[e] = (uint32_t)a;
    t32[e] = (uint32_t)b;
  }
}

__global__ void check_u32_edges(const uint32_t* __restrict__ s, const uint32_t* __restrict__ t,
                                uint64_t m, uint64_t n, unsigned long long* __restrict__ bad) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    if (s[e] >= n) atomicMin(bad, (unsigned long long)(2 * e));
    else if (t[e] >= n) atomicMin(bad, (unsigned long long)(2 * e + 1));
  }
}

// First weight that is not finite (mode 0) or negative (mode 1).
__global__ void first_bad_weight(const double* __restrict__ w, uint64_t m, int mode,
                                 unsigned long long* __restrict__ bad) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    double x = w[e];
    bool b = mode == 0 ? !isfinite(x) : x < 0.0;
    if (b) atomicMin(bad, (unsigned long long)e);
  }
}

__global__ void widen_weights(const float* __restrict__ w32, uint64_t m, double* __restrict__ w) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x)
    w[e] = (double)w32[e];
}

// Degree or strength per node from CSR rows (metrics/degree.rs:41-73): an
// undirected loop counts twice, a directed loop once in each direction;
// loops == 0 skips loops. Integer counts are exact in any order.
__global__ void degree_rows(const uint32_t* __restrict__ off1, const uint32_t* __restrict__ tgt1,
                            const double* __restrict__ w1, const uint32_t* __restrict__ off2,
                            const uint32_t* __restrict__ tgt2, const double* __restrict__ w2,
                            uint32_t n, int undirected, int loops, double* __restrict__ out) {
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
    double s = 0.0;
    for (uint32_t k = off1[v]; k < off1[v + 1]; ++k) {
      double x = w1 ? w1[k] : 1.0;
      if (tgt1[k] == v) {
        if (!loops) continue;
        if (undirected) x += x;
      }
      s += x;
    }
    if (off2) {
      for (uint32_t k = off2[v]; k < off2[v + 1]; ++k) {
        double x = w2 ? w2[k] : 1.0;
        if (tgt2[k] == v && !loops) continue;
        s += x;
      }
    }
    out[v] = s;
  }
}

// ---- simplify (crates/engine/src/metrics/topography.rs:96-141): the
// adjacency-matrix reading of a graph. Loops are dropped; every arc (for an
// undirected result every unordered pair, as (smaller, larger)) is kept
// once, sorted by (from, to), with the largest (keep 0) or smallest (keep 1)
// weight of its parallel edges. Keys pack (from << tb) | to, with the
// sentinel n << tb (after every real key) for a loop.
__global__ void simplify_keys(const uint32_t* __restrict__ src, const uint32_t* __restrict__ tgt,
                              uint64_t m, int directed, int tb, uint64_t sentinel,
                              uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = src[e], b = tgt[e];
    uint64_t k = sentinel;
    if (a != b) {
      const bool keep_order = directed || a < b;
      k = ((uint64_t)(keep_order ? a : b) << tb) | (uint64_t)(keep_order ? b : a);
    }
    keys[e] = k;
    idx[e] = (uint32_t)e;
  }
}

__device__ __forceinline__ bool simplify_head(const uint64_t* keys, uint64_t i, uint64_t sentinel) {
  return keys[i] != sentinel && (i == 0 || keys[i] != keys[i - 1]);
}

__global__ void simplify_heads(const uint64_t* __restrict__ keys, uint64_t m, uint64_t sentinel,
                               uint32_t* __restrict__ head) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x)
    head[i] = simplify_head(keys, i, sentinel) ? 1u : 0u;
}

// One thread per run of equal keys (at its head): the pair and the run's
// largest or smallest weight.
__global__ void simplify_emit(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ idx,
                              const uint32_t* __restrict__ pos, uint64_t m, uint64_t sentinel,
                              int tb, const double* __restrict__ w, int keep_min,
                              uint32_t* __restrict__ out_src, uint32_t* __restrict__ out_tgt,
                              double* __restrict__ out_w) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
       i += (uint64_t)gridDim.x * blockDim.x) {
    if (!simplify_head(keys, i, sentinel)) continue;
    const uint64_t k = keys[i];
    const uint32_t p = pos[i];
    out_src[p] = (uint32_t)(k >> tb);
    out_tgt[p] = (uint32_t)(k & ((1ull << tb) - 1));
    if (w) {
      double x = w[idx[i]];
      for (uint64_t j = i + 1; j < m && keys[j] == k; ++j) {
        const double y = w[idx[j]];
        x = keep_min ? fmin(x, y) : fmax(x, y);
      }
      out_w[p] = x;
    }
  }
}

// First edge whose two ends have the same node type.
__global__ void same_mode_edge(const uint32_t* __restrict__ src, const uint32_t* __restrict__ tgt,
                               uint64_t m, const uint8_t* __restrict__ type,
                               unsigned long long* __restrict__ bad) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x)
    if (type[src[e]] == type[tgt[e]]) atomicMin(bad, (unsigned long long)e);
}

unsigned long long read_u64(const unsigned long long* d, cudaStream_t s) {
  unsigned long long h = 0;
  KNB_CUDA(cudaMemcpyAsync(&h, d, 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  return h;
}

const uint64_t NONE = ~0ull;

// Finishes a handle whose device edge arrays (src, tgt, optional w) are set.
void finish_build(knb::GraphHandleImpl& g, cudaStream_t s) {
  if (g.directed) {
    knb::build_csr(g.n, g.m, g.src.get(), g.tgt.get(), nullptr, g.weighted ? g.w.get() : nullptr,
                   &g.out, s);
    knb::build_csr(g.n, g.m, g.tgt.get(), g.src.get(), nullptr, g.weighted ? g.w.get() : nullptr,
                   &g.inc, s);
  } else {
    knb::build_undirected(g.n, g.m, g.src.get(), g.tgt.get(), g.weighted ? g.w.get() : nullptr,
                          &g.out, s);
  }
}

void check_nonnegative(knb::GraphHandleImpl& g, const char* what, cudaStream_t s) {
  if (!g.weighted) throw Error("the graph has no edge weights");
  knb::DevBuf<unsigned long long> bad(1);
  KNB_CUDA(cudaMemsetAsync(bad.get(), 0xFF, 8, s));
  if (g.m) {
    first_bad_weight<<<knb::grid_for(g.m, 256), 256, 0, s>>>(g.w.get(), g.m, 1, bad.get());
    KNB_LAUNCH("first_bad_weight");
  }
  uint64_t e = read_u64(bad.get(), s);
  if (e != NONE) {
    double w = 0;
    KNB_CUDA(cudaMemcpy(&w, g.w.get() + e, 8, cudaMemcpyDeviceToHost));
    throw Error("edge " + std::to_string(e) + " has negative weight " + fmt_g(w) + "; " + what +
                " requires non-negative weights");
  }
}

}  // namespace

// ======================================================================= C ABI
extern "C" {

int32_t net_graph_new(int64_t n, const int64_t* src, const int64_t* tgt, const double* weights,
                      int64_t m, int32_t directed, GraphHandle** out, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    if (n < 0 || m < 0) throw Error("negative node or edge count");
    if ((uint64_t)n > 0xFFFFFFFFull)
      throw Error("node count (" + std::to_string(n) + ") exceeds the supported maximum");
    if (!out) throw Error("output handle pointer is null");
    cudaStream_t s = knb::thread_stream();
    auto h = std::make_unique<GraphHandle>();
    knb::GraphHandleImpl& g = h->g;
    g.n = (uint32_t)n;
    g.m = (uint64_t)m;
    g.directed = directed != 0;
    g.weighted = weights != nullptr;
    KNB_CUDA(cudaGetDevice(&g.device));
    knb::DevBuf<unsigned long long> bad(1);
    if (g.weighted) {
      if ((uint64_t)m > 0xFFFFFFFFull / 2)
        throw Error("edge count (" + std::to_string(m) + ") exceeds the supported maximum");
      g.w.alloc(std::max<uint64_t>(g.m, 1));
      if (m) KNB_CUDA(cudaMemcpyAsync(g.w.get(), weights, m * 8, cudaMemcpyHostToDevice, s));
      KNB_CUDA(cudaMemsetAsync(bad.get(), 0xFF, 8, s));
      if (m) {
        first_bad_weight<<<knb::grid_for(m, 256), 256, 0, s>>>(g.w.get(), m, 0, bad.get());
        KNB_LAUNCH("first_bad_weight");
      }
      uint64_t e = read_u64(bad.get(), s);
      if (e != NONE)
        throw Error("edge " + std::to_string(e) + " has a missing, NaN, or infinite weight");
    }
    if ((uint64_t)m > 0xFFFFFFFFull / 2)
      throw Error("edge count (" + std::to_string(m) + ") exceeds the supported maximum");
    g.src.alloc(std::max<uint64_t>(g.m, 1));
    g.tgt.alloc(std::max<uint64_t>(g.m, 1));
    if (m) {
      knb::DevBuf<int64_t> s64(m), t64(m);
      KNB_CUDA(cudaMemcpyAsync(s64.get(), src, m * 8, cudaMemcpyHostToDevice, s));
      KNB_CUDA(cudaMemcpyAsync(t64.get(), tgt, m * 8, cudaMemcpyHostToDevice, s));
      KNB_CUDA(cudaMemsetAsync(bad.get(), 0xFF, 8, s));
      convert_edges<<<knb::grid_for(m, 256), 256, 0, s>>>(s64.get(), t64.get(), m, (uint64_t)n,
                                                          g.src.get(), g.tgt.get(), bad.get());
      KNB_LAUNCH("convert_edges");
      uint64_t b = read_u64(bad.get(), s);
      if (b != NONE) {
        uint64_t e = b / 2;
        int64_t node = (b & 1) ? tgt[e] : src[e];
        throw Error("edge " + std::to_string(e) + " refers to node index " + std::to_string(node) +
                    ", but valid indices are 0.." + std::to_string(n));
      }
    }
    finish_build(g, s);
    *out = h.release();
  });
}

void net_graph_free(GraphHandle* h) { delete h; }

int64_t net_graph_node_count(const GraphHandle* h) { return h ? (int64_t)h->g.n : -1; }

int64_t net_graph_edge_count(const GraphHandle* h) { return h ? (int64_t)h->g.m : -1; }

int32_t net_degree(const GraphHandle* h, int32_t mode, int32_t loops, int32_t weighted,
                   double* out, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    if (mode < 1 || mode > 3) throw Error("unknown degree mode code " + std::to_string(mode));
    if (weighted && !g.weighted) throw Error("the graph has no edge weights");
    if (g.n == 0) return;
    cudaStream_t s = knb::thread_stream();
    knb::DevBuf<double> d(g.n);
    const knb::DevCsr* a = &g.out;
    const knb::DevCsr* b = nullptr;
    if (g.directed) {
      if (mode == 2) a = &g.inc;
      if (mode == 3) b = &g.inc;
    }
    degree_rows<<<knb::grid_for(g.n, 128), 128, 0, s>>>(
        a->off.get(), a->tgt.get(), weighted ? a->w.get() : nullptr, b ? b->off.get() : nullptr,
        b ? b->tgt.get() : nullptr, (b && weighted) ? b->w.get() : nullptr, g.n, g.directed ? 0 : 1,
        loops != 0, d.get());
    KNB_LAUNCH("degree_rows");
    KNB_CUDA(cudaMemcpyAsync(out, d.get(), (size_t)g.n * 8, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
  });
}

static int32_t pagerank_impl(const GraphHandle* h, double damping, int32_t directed,
                             int32_t weighted, const double* personalization, int pers_dev,
                             int32_t dangling, int32_t loops, double tol, int64_t max_iter,
                             int32_t precision, double* out, int out_dev, NetSolveInfo* info,
                             char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    if (dangling != 0 && dangling != 1)
      throw Error("unknown dangling-node code " + std::to_string(dangling));
    if (loops < 0 || loops > 2) throw Error("unknown self-loop weight code " + std::to_string(loops));
    if (precision < 0 || precision > 2)
      throw Error("unknown precision code " + std::to_string(precision));
    knb::PagerankParams p;
    p.damping = damping;
    p.directed = directed != 0;
    p.weighted = weighted != 0;
    p.dangling = dangling;
    p.loops = loops;
    p.tol = tolerance(tol);
    p.max_iter = max_iter > 0 ? max_iter : 10000;
    p.precision = precision;
    if (!(damping >= 0.0 && damping <= 1.0))
      throw Error("damping is " + fmt_g(damping) + "; it must be between 0 and 1");
    if (g.n == 0) return;
    cudaStream_t s = knb::thread_stream();
    if (p.weighted) check_nonnegative(g, "PageRank", s);
    if (personalization) {
      // checked and rescaled on the device (pagerank.cu, normalize_personalization)
      p.personalization = personalization;
      p.pers_on_device = pers_dev != 0;
    }
    // A small graph's FP64 solve (teleport vector, if any, in host memory)
    // runs as a packed batch of one graph: one launch does every iteration
    // on the device (a cluster of CTAs splits it from 4096 nodes), where the
    // sweep path would launch a few kernels per iteration that each take
    // microseconds. The packed path checks a teleport vector with the same
    // messages.
    const knb::Tuning& tu = knb::tuning();
    if (precision == 0 && (!personalization || !pers_dev) && tu.variant == 0 &&
        tu.small_edges > 0 && (int64_t)g.m <= tu.small_edges) {
      const int64_t off[2] = {0, (int64_t)g.n};
      int64_t iters = 0;
      knb::EgoInput in;
      in.count = 1;
      in.node_offsets = off;
      in.damping = p.damping;
      in.directed = p.directed;
      in.weighted = p.weighted;
      in.dangling = dangling;
      in.loops = loops;
      in.tol = p.tol;
      in.max_iter = p.max_iter;
      in.personalization = personalization;
      in.out_on_device = out_dev != 0;
      in.iterations_out = &iters;
      knb::EgoResult r;
      knb::pagerank_graphs(g, in, out, &r, s);
      if (info) {
        memset(info, 0, sizeof(*info));
        info->iterations = iters;
        info->change = r.change;
        info->seconds = r.seconds;
        info->converged = 1;
        info->kernel_launches = 1;
        info->sweep_kernel = 0;  // no sweep kernel: the packed-graph launch
        info->long_row = r.instantiations;
        info->hot_columns = r.cluster;
      }
      return;
    }
    knb::PagerankInfo pi;
    knb::pagerank(g, p, out, out_dev != 0, &pi, s);
    if (info) {
      memset(info, 0, sizeof(*info));
      info->iterations = pi.iterations;
      info->iterations_fp32 = pi.iterations_fp32;
      info->change = pi.change;
      info->seconds = pi.seconds;
      info->converged = pi.converged;
      info->kernel_launches = pi.kernel_launches;
      info->sweep_kernel = pi.sweep_kernel;
      info->long_row = pi.long_row;
      info->hot_columns = pi.hot_columns;
    }
  });
}

int32_t net_pagerank(const GraphHandle* h, double damping, int32_t directed, int32_t weighted,
                     const double* personalization, int32_t dangling, int32_t loops, double tol,
                     int64_t max_iter, int32_t threads, double* out, char* err, size_t err_len) {
  (void)threads;  // results never depend on it; the device decides the parallelism
  return pagerank_impl(h, damping, directed, weighted, personalization, 0, dangling, loops, tol,
                       max_iter, 0, out, 0, nullptr, err, err_len);
}

int32_t net_pagerank_ex(const GraphHandle* h, double damping, int32_t directed, int32_t weighted,
                        const double* personalization, int32_t dangling, int32_t loops, double tol,
                        int64_t max_iter, int32_t precision, double* out, NetSolveInfo* info,
                        char* err, size_t err_len) {
  return pagerank_impl(h, damping, directed, weighted, personalization, 0, dangling, loops, tol,
                       max_iter, precision, out, 0, info, err, err_len);
}

int32_t net_pagerank_device(const GraphHandle* h, double damping, int32_t directed,
                            int32_t weighted, const double* d_personalization, int32_t dangling,
                            int32_t loops, double tol, int64_t max_iter, int32_t precision,
                            double* d_out, NetSolveInfo* info, char* err, size_t err_len) {
  return pagerank_impl(h, damping, directed, weighted, d_personalization, 1, dangling, loops, tol,
                       max_iter, precision, d_out, 1, info, err, err_len);
}

static int32_t eigen_impl(const GraphHandle* h, int32_t mode, int32_t weighted, int32_t scale,
                          int32_t loops, double tol, int64_t max_iter, int32_t precision,
                          double* out, double* eigenvalue, int32_t* connected, NetSolveInfo* info,
                          char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    // Codes decoded first, as the reference's C wrapper does
    // (crates/capi/src/topography.rs:225-240).
    if (mode < 1 || mode > 3) throw Error("unknown degree mode code " + std::to_string(mode));
    if (scale != 0 && scale != 1)
      throw Error("unknown eigenvector scale code " + std::to_string(scale));
    if (loops < 0 || loops > 2) throw Error("unknown self-loop weight code " + std::to_string(loops));
    if (precision != 0 && precision != 1)
      throw Error("unknown precision code " + std::to_string(precision));
    knb::EigenParams p;
    p.mode = mode;
    p.weighted = weighted != 0;
    p.scale = scale;
    p.loops = loops;
    p.tol = tolerance(tol);
    p.max_iter = max_iter > 0 ? max_iter : 10000;
    p.precision = precision;
    cudaStream_t s = knb::thread_stream();
    if (g.n > 0 && p.weighted) check_nonnegative(g, "eigenvector centrality", s);
    knb::EigenResult r;
    knb::eigenvector(g, p, out, &r, s);
    if (eigenvalue) *eigenvalue = r.eigenvalue;
    if (connected) *connected = r.connected ? 1 : 0;
    if (info) {
      memset(info, 0, sizeof(*info));
      info->iterations = r.matvecs;
      info->iterations_fp32 = r.matvecs_fp32;
      info->seconds = r.seconds;
      info->converged = 1;
      info->kernel_launches = r.kernel_launches;
      info->eigenvalue = r.eigenvalue;
      info->connected = r.connected ? 1 : 0;
    }
  });
}

// net_katz and net_bonacich_power: codes decoded and options checked in the
// order of crates/capi/src/spectral.rs:107-179 and spectral.rs:365-385,
// 596-611.
static void series_codes(int32_t mode, int32_t loops) {
  if (mode < 1 || mode > 3) throw Error("unknown degree mode code " + std::to_string(mode));
  if (loops < 0 || loops > 2) throw Error("unknown self-loop weight code " + std::to_string(loops));
}

int32_t net_katz(const GraphHandle* h, double alpha, const double* beta, int64_t beta_len,
                 int32_t mode, int32_t weighted, int32_t loops, int32_t normalized, double tol,
                 int64_t max_iter, int32_t threads, double* out, char* err, size_t err_len) {
  (void)threads;
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    if (beta_len < 0) throw Error("beta length must be non-negative");
    if (beta_len > 0 && !beta) throw Error("beta is NULL");
    series_codes(mode, loops);
    knb::SeriesParams p;
    p.mode = mode;
    p.weighted = weighted != 0;
    p.loops = loops;
    p.tol = tolerance(tol);
    p.max_iter = max_iter > 0 ? max_iter : 10000;
    if (!std::isfinite(alpha) || alpha < 0.0)
      throw Error("alpha is " + fmt_g(alpha) +
                  "; it must be a nonnegative number below 1 / lambda_max");
    const uint32_t n = g.n;
    std::vector<double> b;
    if (beta_len == 1) b.assign(n, beta[0]);
    else if ((uint64_t)beta_len == n) b.assign(beta, beta + n);
    else
      throw Error("beta: expected length " + std::to_string(n) + ", found " +
                  std::to_string(beta_len));
    for (double v : b)
      if (!std::isfinite(v)) throw Error("beta must be finite");
    if (n == 0) return;
    cudaStream_t s = knb::thread_stream();
    if (p.weighted) check_nonnegative(g, "Katz centrality", s);
    knb::SeriesResult r;
    knb::katz(g, alpha, b, normalized != 0, p, out, &r, s);
  });
}

int32_t net_bonacich_power(const GraphHandle* h, double exponent, int32_t mode, int32_t weighted,
                           int32_t loops, int32_t rescale, double tol, int64_t max_iter,
                           int32_t threads, double* out, char* err, size_t err_len) {
  (void)threads;
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    series_codes(mode, loops);
    knb::SeriesParams p;
    p.mode = mode;
    p.weighted = weighted != 0;
    p.loops = loops;
    p.tol = tolerance(tol);
    p.max_iter = max_iter > 0 ? max_iter : 10000;
    if (!std::isfinite(exponent)) throw Error("the exponent must be finite");
    if (g.n == 0) return;
    cudaStream_t s = knb::thread_stream();
    if (p.weighted) check_nonnegative(g, "power centrality", s);
    knb::SeriesResult r;
    knb::bonacich_power(g, exponent, rescale != 0, p, out, &r, s);
  });
}

// net_hits: codes decoded as crates/capi/src/spectral.rs:189-230.
int32_t net_hits(const GraphHandle* h, int32_t weighted, int32_t loops, int32_t scale, double tol,
                 int64_t max_iter, int32_t threads, double* hubs, double* authorities,
                 double* value, int32_t* unique, char* err, size_t err_len) {
  (void)threads;
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    if (loops < 0 || loops > 2) throw Error("unknown self-loop weight code " + std::to_string(loops));
    if (scale < 0 || scale > 2)
      throw Error("unknown hub and authority scale code " + std::to_string(scale));
    knb::HitsParams p;
    p.weighted = weighted != 0;
    p.loops = loops;
    p.scale = scale;
    p.tol = tolerance(tol);
    p.max_iter = max_iter > 0 ? max_iter : 10000;
    cudaStream_t s = knb::thread_stream();
    if (p.weighted) check_nonnegative(g, "hub and authority scores", s);
    double v = 0.0;
    int u = 0;
    if (g.n == 0) {
      v = 0.0;
      u = 0;
    } else {
      knb::hits(g, p, hubs, authorities, &v, &u, s);
    }
    if (value) *value = v;
    if (unique) *unique = u;
  });
}

int32_t net_eigenvector(const GraphHandle* h, int32_t mode, int32_t weighted, int32_t scale,
                        int32_t loops, double tol, int64_t max_iter, int32_t threads, double* out,
                        double* eigenvalue, int32_t* connected, char* err, size_t err_len) {
  (void)threads;
  return eigen_impl(h, mode, weighted, scale, loops, tol, max_iter, 0, out, eigenvalue, connected,
                    nullptr, err, err_len);
}

int32_t net_eigenvector_ex(const GraphHandle* h, int32_t mode, int32_t weighted, int32_t scale,
                           int32_t loops, double tol, int64_t max_iter, int32_t precision,
                           double* out, double* eigenvalue, int32_t* connected,
                           NetSolveInfo* info, char* err, size_t err_len) {
  return eigen_impl(h, mode, weighted, scale, loops, tol, max_iter, precision, out, eigenvalue,
                    connected, info, err, err_len);
}

int32_t net_graph_simplify(const GraphHandle* h, int32_t undirected, int32_t keep,
                           GraphHandle** out, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    // ParallelWeight::from_code (crates/engine/src/metrics/topography.rs:86-96)
    if (keep != 0 && keep != 1)
      throw Error("unknown parallel-edge weight code " + std::to_string(keep));
    if (!out) throw Error("output handle pointer is null");
    cudaStream_t s = knb::thread_stream();
    const bool directed = g.directed && !undirected;
    const uint64_t m = g.m;
    int tb = 0;
    while (tb < 32 && (1ull << tb) < (uint64_t)g.n) ++tb;
    int hb = 0;
    while (hb < 33 && (1ull << hb) < (uint64_t)g.n + 1) ++hb;
    const uint64_t sentinel = (uint64_t)g.n << tb;
    knb::DevBuf<uint64_t> keys(std::max<uint64_t>(m, 1));
    knb::DevBuf<uint32_t> idx(std::max<uint64_t>(m, 1)), pos(std::max<uint64_t>(m, 1));
    uint64_t mo = 0;
    if (m) {
      const unsigned gm = knb::grid_for(m, 256);
      simplify_keys<<<gm, 256, 0, s>>>(g.src.get(), g.tgt.get(), m, directed ? 1 : 0, tb, sentinel,
                                       keys.get(), idx.get());
      KNB_LAUNCH("simplify_keys");
      knb::radix_sort(keys.get(), idx.get(), m, tb + hb, s);
      simplify_heads<<<gm, 256, 0, s>>>(keys.get(), m, sentinel, pos.get());
      KNB_LAUNCH("simplify_heads");
      mo = knb::exclusive_scan<uint32_t>(pos.get(), pos.get(), m, s);
    }
    knb::DevBuf<uint32_t> os(std::max<uint64_t>(mo, 1)), ot(std::max<uint64_t>(mo, 1));
    knb::DevBuf<double> ow(g.weighted ? std::max<uint64_t>(mo, 1) : 0);
    if (mo) {
      simplify_emit<<<knb::grid_for(m, 256), 256, 0, s>>>(
          keys.get(), idx.get(), pos.get(), m, sentinel, tb, g.weighted ? g.w.get() : nullptr,
          keep, os.get(), ot.get(), g.weighted ? ow.get() : nullptr);
      KNB_LAUNCH("simplify_emit");
    }
    char e2[512] = {0};
    if (net_graph_new_device((int64_t)g.n, os.get(), ot.get(), nullptr,
                             g.weighted ? ow.get() : nullptr, (int64_t)mo, directed ? 1 : 0, out,
                             e2, sizeof e2))
      throw Error(e2);
  });
}

int32_t net_twomode_eigenvector(const GraphHandle* h, const int32_t* types, double tol,
                                int64_t max_iter, int32_t threads, double* out,
                                double* eigenvalue, int32_t* connected, char* err,
                                size_t err_len) {
  (void)threads;
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    // types_from, check_types (crates/capi/src/twomode.rs:50-66,
    // crates/engine/src/metrics/bipartite.rs:93-111)
    if (!types) throw Error("node types are missing");
    const uint32_t n = g.n;
    std::vector<uint8_t> t(std::max<uint32_t>(n, 1), 0);
    for (uint32_t v = 0; v < n; ++v) {
      if (types[v] != 0 && types[v] != 1)
        throw Error("node " + std::to_string(v) + " has type code " + std::to_string(types[v]) +
                    "; use 0 for the first mode and 1 for the second");
      t[v] = (uint8_t)types[v];
    }
    const double tl = tolerance(tol);
    const int64_t mi = max_iter > 0 ? max_iter : 10000;
    cudaStream_t s = knb::thread_stream();
    if (g.m) {
      knb::DevBuf<uint8_t> td(std::max<uint32_t>(n, 1));
      knb::DevBuf<unsigned long long> bad(1);
      KNB_CUDA(cudaMemcpyAsync(td.get(), t.data(), n, cudaMemcpyHostToDevice, s));
      KNB_CUDA(cudaMemsetAsync(bad.get(), 0xFF, 8, s));
      same_mode_edge<<<knb::grid_for(g.m, 256), 256, 0, s>>>(g.src.get(), g.tgt.get(), g.m,
                                                             td.get(), bad.get());
      KNB_LAUNCH("same_mode_edge");
      const uint64_t e = read_u64(bad.get(), s);
      if (e != NONE) {
        uint32_t a = 0, b = 0;
        KNB_CUDA(cudaMemcpyAsync(&a, g.src.get() + e, 4, cudaMemcpyDeviceToHost, s));
        KNB_CUDA(cudaMemcpyAsync(&b, g.tgt.get() + e, 4, cudaMemcpyDeviceToHost, s));
        KNB_CUDA(cudaStreamSynchronize(s));
        throw Error("edge " + std::to_string(e) + " joins nodes " + std::to_string(a) + " and " +
                    std::to_string(b) +
                    ", which are in the same mode; in a two-mode network every edge joins the "
                    "two modes");
      }
    }
    // the binary affiliation graph (bipartite.rs:113-116), then eigenvector
    // centrality with direction ignored, unweighted, unit scale, loops
    // ignored; each mode's half scaled to length 1 (bipartite.rs:288-336)
    GraphHandle* a = nullptr;
    char e2[512] = {0};
    if (net_graph_simplify(h, 1, 0, &a, e2, sizeof e2)) throw Error(e2);
    std::unique_ptr<GraphHandle> own(a);
    knb::EigenParams p;
    p.mode = 3;
    p.weighted = false;
    p.scale = 1;
    p.loops = 2;
    p.tol = tl;
    p.max_iter = mi;
    knb::EigenResult r;
    std::vector<double> x(std::max<uint32_t>(n, 1));
    knb::eigenvector(a->g, p, x.data(), &r, s);
    if (a->g.m == 0) {
      for (uint32_t v = 0; v < n; ++v) out[v] = std::numeric_limits<double>::quiet_NaN();
      if (eigenvalue) *eigenvalue = 0.0;
      if (connected) *connected = r.connected ? 1 : 0;
      return;
    }
    for (uint8_t mode = 0; mode < 2; ++mode) {
      double ss = 0.0;
      for (uint32_t v = 0; v < n; ++v)
        if (t[v] == mode) ss += x[v] * x[v];
      const double norm = std::sqrt(ss);
      if (norm > 0.0)
        for (uint32_t v = 0; v < n; ++v)
          if (t[v] == mode) x[v] /= norm;
    }
    memcpy(out, x.data(), (size_t)n * 8);
    if (eigenvalue) *eigenvalue = r.eigenvalue;
    if (connected) *connected = r.connected ? 1 : 0;
  });
}

int32_t net_leading_eigen(const GraphHandle* h, int32_t weighted, int64_t* membership, double* q,
                          int64_t* splits, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    // require_undirected, MAX_NODES, additive_weights
    // (crates/engine/src/metrics/partition.rs:52-70, partition/leading_eigen.rs:57-68)
    if (g.directed)
      throw Error("The leading eigenvector method is defined here for undirected networks only; "
                  "build the network as undirected first");
    if (g.n > 3000)
      throw Error("the leading eigenvector method uses a dense eigendecomposition and is limited "
                  "to 3000 nodes");
    cudaStream_t s = knb::thread_stream();
    if (weighted) check_nonnegative(g, "modularity", s);
    knb::leading_eigen(g, weighted != 0, membership, q, splits, nullptr, s);
  });
}

int32_t net_components(const GraphHandle* h, int32_t kind, int32_t* membership, int64_t* count,
                       char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    // ComponentKind::from_code (crates/engine/src/metrics/topography.rs:152-163)
    if (kind != 0 && kind != 1) throw Error("unknown component kind code " + std::to_string(kind));
    cudaStream_t s = knb::thread_stream();
    knb::Comps c = kind == 1 && g.directed ? knb::strong_components(g, nullptr, false, nullptr, s)
                                           : knb::weak_components(g, s);
    for (uint32_t v = 0; v < g.n; ++v) {
      if (c.membership[v] > (uint32_t)INT32_MAX)
        throw Error("component count " + std::to_string(c.membership[v]) + " is too large");
      membership[v] = (int32_t)c.membership[v];
    }
    *count = (int64_t)c.count();
  });
}

int32_t net_centralization(const GraphHandle* h, int32_t measure, int32_t mode, int32_t loops,
                           int32_t normalized, int32_t convention, int32_t threads, double* out,
                           char* err, size_t err_len) {
  (void)threads;
  (void)loops;  // degree centralization only
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    // codes, then the convention and measure rules
    // (crates/engine/src/metrics/topography.rs:320-334,376-387,475-498)
    if (measure < 0 || measure > 3)
      throw Error("unknown centralization measure code " + std::to_string(measure));
    if (mode < 1 || mode > 3) throw Error("unknown degree mode code " + std::to_string(mode));
    if (convention < 0 || convention > 3)
      throw Error("unknown convention code " + std::to_string(convention));
    static const char* names[] = {"igraph", "NetworkX", "sna", "UCINET"};
    if (convention == 1)
      throw Error("NetworkX has no centralization index; use the igraph, sna, or UCINET convention");
    if (measure != 3)
      throw Error("degree, betweenness and closeness centralization are outside this library, "
                  "which provides the spectral measures only (measure 3, eigenvector)");
    if (convention != 0)
      throw Error(std::string("eigenvector centralization is provided for the igraph convention "
                              "only, not ") + names[convention]);
    if (g.directed && mode != 3)
      throw Error("eigenvector centralization is provided with direction ignored (mode \"all\") only");
    const uint32_t n = g.n;
    if (n == 0) {
      *out = std::numeric_limits<double>::quiet_NaN();
      return;
    }
    // eigenvector centrality, direction ignored, unweighted, scaled to max
    // 1, loops twice, default tolerance and cap; then Freeman's index
    // n max - sum, over n - 2 when normalized (topography.rs:446-472,512-560)
    knb::EigenParams p;
    p.mode = 3;
    p.weighted = false;
    p.scale = 0;
    p.loops = 0;
    p.tol = 1e-12;
    p.max_iter = 10000;
    std::vector<double> x(n);
    knb::EigenResult r;
    knb::eigenvector(g, p, x.data(), &r, knb::thread_stream());
    double mx = -std::numeric_limits<double>::infinity(), total = 0.0;
    bool nan = false;
    for (double v : x) {
      mx = std::fmax(mx, v);
      total += v;
      nan = nan || std::isnan(v);
    }
    if (nan) mx = std::numeric_limits<double>::quiet_NaN();
    const double raw = (double)n * mx - total;
    if (!normalized) {
      *out = raw;
      return;
    }
    const double tmax = n < 3 ? std::numeric_limits<double>::quiet_NaN() : (double)n - 2.0;
    *out = raw / tmax;
  });
}

int32_t net_generate_rmat(int32_t scale, int64_t edge_factor, double a, double b, double c,
                          uint64_t seed, int32_t clean, int32_t symmetrize, int32_t lognormal,
                          uint64_t wseed, GraphHandle** out, int64_t* m_out, char* err,
                          size_t err_len) {
  return guard(err, err_len, [&] {
    if (edge_factor < 0) throw Error("edge factor must be non-negative");
    cudaStream_t s = knb::thread_stream();
    knb::RmatEdges e = knb::generate_rmat(scale, (uint64_t)edge_factor, a, b, c, seed, clean != 0,
                                          symmetrize != 0, lognormal != 0, wseed, s);
    auto h = std::make_unique<GraphHandle>();
    knb::GraphHandleImpl& g = h->g;
    g.n = e.n;
    g.m = e.m;
    g.directed = symmetrize == 0;
    g.weighted = lognormal != 0;
    KNB_CUDA(cudaGetDevice(&g.device));
    g.src = std::move(e.src);
    g.tgt = std::move(e.tgt);
    if (g.weighted) {
      g.w.alloc(std::max<uint64_t>(g.m, 1));
      if (g.m) {
        widen_weights<<<knb::grid_for(g.m, 256), 256, 0, s>>>(e.w32.get(), g.m, g.w.get());
        KNB_LAUNCH("widen_weights");
      }
    }
    finish_build(g, s);
    if (m_out) *m_out = (int64_t)g.m;
    *out = h.release();
  });
}

static int32_t batch_impl(const GraphHandle* h, double damping, int32_t directed, int32_t weighted,
                          const double* personalization, int64_t batch, int32_t dangling,
                          int32_t loops, double tol, int64_t max_iter, int32_t precision,
                          int on_device, double* out, NetBatchInfo* info, char* err,
                          size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    if (dangling != 0 && dangling != 1)
      throw Error("unknown dangling-node code " + std::to_string(dangling));
    if (loops < 0 || loops > 2) throw Error("unknown self-loop weight code " + std::to_string(loops));
    if (precision != 0 && precision != 1)
      throw Error("unknown precision code " + std::to_string(precision));
    if (batch < 0 || batch > 0xFFFFFFFFll) throw Error("batch size out of range");
    if (!personalization && batch > 0)
      throw Error("a batch needs one personalization vector per column");
    knb::BatchParams p;
    p.damping = damping;
    p.directed = directed != 0;
    p.weighted = weighted != 0;
    p.dangling = dangling;
    p.loops = loops;
    p.tol = tolerance(tol);
    p.max_iter = max_iter > 0 ? max_iter : 10000;
    p.precision = precision;
    p.B = (uint32_t)batch;
    p.on_device = on_device != 0;
    const knb::Tuning& tu = knb::tuning();
    p.switch_factor = tu.switch_factor;
    p.switch_floor = tu.switch_floor;
    if (!(damping >= 0.0 && damping <= 1.0))
      throw Error("damping is " + fmt_g(damping) + "; it must be between 0 and 1");
    if (g.n == 0 || batch == 0) return;
    cudaStream_t s = knb::thread_stream();
    if (p.weighted) check_nonnegative(g, "PageRank", s);
    knb::BatchInfo bi;
    knb::pagerank_batch(g, p, personalization, out, &bi, s);
    if (info) {
      memset(info, 0, sizeof(*info));
      info->seconds = bi.seconds;
      info->sweeps = bi.sweeps;
      info->sweeps_fp32 = bi.sweeps_fp32;
      info->column_iterations = bi.column_iterations;
      info->max_column_iterations = bi.max_column_iterations;
      info->kernel_launches = bi.kernel_launches;
      info->sweep_seconds = bi.sweep_seconds;
      info->column_iterations_fp32 = bi.column_iterations_fp32;
      info->refined = bi.refined;
    }
  });
}

int32_t net_pagerank_batch(const GraphHandle* h, double damping, int32_t directed,
                           int32_t weighted, const double* personalization, int64_t batch,
                           int32_t dangling, int32_t loops, double tol, int64_t max_iter,
                           int32_t precision, double* out, NetBatchInfo* info, char* err,
                           size_t err_len) {
  return batch_impl(h, damping, directed, weighted, personalization, batch, dangling, loops, tol,
                    max_iter, precision, 0, out, info, err, err_len);
}

int32_t net_pagerank_batch_device(const GraphHandle* h, double damping, int32_t directed,
                                  int32_t weighted, const double* d_personalization,
                                  int64_t batch, int32_t dangling, int32_t loops, double tol,
                                  int64_t max_iter, int32_t precision, double* d_out,
                                  NetBatchInfo* info, char* err, size_t err_len) {
  return batch_impl(h, damping, directed, weighted, d_personalization, batch, dangling, loops, tol,
                    max_iter, precision, 1, d_out, info, err, err_len);
}

int32_t net_pagerank_graphs(const GraphHandle* h, int64_t count, const int64_t* node_offsets,
                            double damping, int32_t directed, int32_t weighted,
                            const double* personalization, int32_t dangling, int32_t loops,
                            double tol, int64_t max_iter, double* out, int64_t* iterations,
                            NetSolveInfo* info, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    if (dangling != 0 && dangling != 1)
      throw Error("unknown dangling-node code " + std::to_string(dangling));
    if (loops < 0 || loops > 2) throw Error("unknown self-loop weight code " + std::to_string(loops));
    if (count < 1 || count > 0xFFFFFFFll) throw Error("graph count out of range");
    if (!node_offsets) throw Error("graph offsets are null");
    knb::EgoInput in;
    in.count = (uint32_t)count;
    in.node_offsets = node_offsets;
    in.damping = damping;
    in.directed = directed != 0;
    in.weighted = weighted != 0;
    in.dangling = dangling;
    in.loops = loops;
    in.tol = tolerance(tol);
    in.max_iter = max_iter > 0 ? max_iter : 10000;
    in.personalization = personalization;
    in.iterations_out = iterations;
    if (!(damping >= 0.0 && damping <= 1.0))
      throw Error("damping is " + fmt_g(damping) + "; it must be between 0 and 1");
    if (g.n == 0) return;
    cudaStream_t s = knb::thread_stream();
    if (in.weighted) check_nonnegative(g, "PageRank", s);
    knb::EgoResult r;
    knb::pagerank_graphs(g, in, out, &r, s);
    if (info) {
      memset(info, 0, sizeof(*info));
      info->iterations = r.total_iterations;
      info->seconds = r.seconds;
      info->converged = 1;
      info->kernel_launches = 1;
      info->sweep_kernel = r.threads;  // threads per CTA of the packed launch
      info->long_row = r.instantiations;  // instantiations of the operator's launch graph
      info->hot_columns = r.cluster;      // CTAs per cluster that split the large graphs
      info->iterations_fp32 = r.split_graphs;  // graphs split over a cluster
    }
  });
}

int32_t net_generate_gnm(int64_t count, const int64_t* n, const int64_t* m, int32_t directed,
                         int32_t loops, uint64_t seed, int64_t* src, int64_t* tgt, char* err,
                         size_t err_len) {
  return guard(err, err_len, [&] {
    if (count < 0) throw Error("negative graph count");
    for (int64_t k = 0; k < count; ++k)
      if (n[k] < 0 || m[k] < 0) throw Error("negative node or edge count");
    knb::gnm_batch((uint64_t)count, n, m, directed != 0, loops != 0, seed, src, tgt, 0);
  });
}

int32_t net_power_law_sizes(int64_t count, double alpha, double lo, double hi, uint64_t seed,
                            int64_t* out, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    if (count < 0 || !(alpha > 1.0) || !(lo >= 1.0) || !(hi >= lo))
      throw Error("power law needs alpha > 1 and 1 <= lo <= hi");
    knb::power_law_sizes((uint64_t)count, alpha, lo, hi, seed, out);
  });
}

__global__ void first_bad_weight_dev(const double* __restrict__ w, uint64_t m,
                                     unsigned long long* __restrict__ bad) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x)
    if (!isfinite(w[e]) || w[e] < 0.0) atomicMin(bad, (unsigned long long)e);
}

static void check_device_weights(const knb::GraphHandleImpl& g, const double* d_w, cudaStream_t s) {
  if (!d_w) throw Error("the weight vector is null");
  if (!g.m) return;
  knb::DevBuf<unsigned long long> bad(1);
  KNB_CUDA(cudaMemsetAsync(bad.get(), 0xFF, 8, s));
  first_bad_weight_dev<<<knb::grid_for(g.m, 256), 256, 0, s>>>(d_w, g.m, bad.get());
  KNB_LAUNCH("first_bad_weight_dev");
  uint64_t e = read_u64(bad.get(), s);
  if (e != NONE)
    throw Error("edge " + std::to_string(e) +
                " has a negative or non-finite weight; PageRank requires non-negative weights");
}

int32_t net_pagerank_weights_device(const GraphHandle* h, const double* d_weights, double damping,
                                    int32_t directed, const double* d_personalization,
                                    int32_t dangling, int32_t loops, double tol, int64_t max_iter,
                                    int32_t precision, double* d_out, NetSolveInfo* info,
                                    char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    if (dangling != 0 && dangling != 1)
      throw Error("unknown dangling-node code " + std::to_string(dangling));
    if (loops < 0 || loops > 2) throw Error("unknown self-loop weight code " + std::to_string(loops));
    if (precision < 0 || precision > 2)
      throw Error("unknown precision code " + std::to_string(precision));
    if (!(damping >= 0.0 && damping <= 1.0))
      throw Error("damping is " + fmt_g(damping) + "; it must be between 0 and 1");
    if (g.n == 0) return;
    cudaStream_t s = knb::thread_stream();
    check_device_weights(g, d_weights, s);
    knb::PagerankParams p;
    p.damping = damping;
    p.directed = directed != 0;
    p.weighted = true;
    p.personalization = d_personalization;
    p.pers_on_device = true;
    p.dangling = dangling;
    p.loops = loops;
    p.tol = tolerance(tol);
    p.max_iter = max_iter > 0 ? max_iter : 10000;
    p.precision = precision;
    knb::PagerankInfo pi;
    knb::pagerank_weights(g, d_weights, p, d_out, &pi, s);
    if (info) {
      memset(info, 0, sizeof(*info));
      info->iterations = pi.iterations;
      info->iterations_fp32 = pi.iterations_fp32;
      info->change = pi.change;
      info->seconds = pi.seconds;
      info->converged = pi.converged;
      info->kernel_launches = pi.kernel_launches;
      info->sweep_kernel = pi.sweep_kernel;
      info->long_row = pi.long_row;
      info->hot_columns = pi.hot_columns;
    }
  });
}

int32_t net_pagerank_grad_device(const GraphHandle* h, const double* d_weights,
                                 const double* d_scores, const double* d_grad_scores,
                                 double damping, int32_t directed,
                                 const double* d_personalization, int32_t dangling, int32_t loops,
                                 double tol, int64_t max_iter, double* d_grad_weights,
                                 double* d_lambda, NetSolveInfo* info, char* err,
                                 size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    if (dangling != 0 && dangling != 1)
      throw Error("unknown dangling-node code " + std::to_string(dangling));
    if (loops < 0 || loops > 2) throw Error("unknown self-loop weight code " + std::to_string(loops));
    if (!(damping >= 0.0 && damping < 1.0))
      throw Error("damping is " + fmt_g(damping) + "; the adjoint needs 0 <= damping < 1");
    if (!d_scores || !d_grad_scores || !d_grad_weights) throw Error("a device vector is null");
    cudaStream_t s = knb::thread_stream();
    check_device_weights(g, d_weights, s);
    knb::AdjointParams p;
    p.damping = damping;
    p.directed = directed != 0;
    p.dangling = dangling;
    p.loops = loops;
    p.personalization = d_personalization;
    p.tol = tolerance(tol);
    p.max_iter = max_iter > 0 ? max_iter : 10000;
    knb::AdjointInfo ai;
    knb::pagerank_grad(g, d_weights, d_scores, d_grad_scores, p, d_grad_weights, d_lambda, &ai, s);
    if (info) {
      memset(info, 0, sizeof(*info));
      info->iterations = ai.iterations;
      info->change = ai.change;
      info->seconds = ai.seconds;
      info->converged = 1;
      info->kernel_launches = ai.kernel_launches;
    }
  });
}

int64_t net_graph_arc_count(const GraphHandle* h, int32_t which) {
  if (!h) return -1;
  const knb::GraphHandleImpl& g = h->g;
  if (which == 1) return (int64_t)g.in_rows().arcs;
  return (int64_t)g.out.arcs;
}

int32_t net_graph_csr(const GraphHandle* h, int32_t which, uint32_t* off, uint32_t* tgt,
                      uint32_t* edge, double* w, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    cudaStream_t s = knb::thread_stream();
    const knb::DevCsr* c = which == 1 ? &g.in_rows() : which == 2 ? &g.undirected_rows(s) : &g.out;
    KNB_CUDA(cudaMemcpyAsync(off, c->off.get(), ((size_t)g.n + 1) * 4, cudaMemcpyDeviceToHost, s));
    if (c->arcs) {
      if (tgt) KNB_CUDA(cudaMemcpyAsync(tgt, c->tgt.get(), c->arcs * 4, cudaMemcpyDeviceToHost, s));
      if (edge) KNB_CUDA(cudaMemcpyAsync(edge, c->edge.get(), c->arcs * 4, cudaMemcpyDeviceToHost, s));
      if (w && g.weighted)
        KNB_CUDA(cudaMemcpyAsync(w, c->w.get(), c->arcs * 8, cudaMemcpyDeviceToHost, s));
    }
    KNB_CUDA(cudaStreamSynchronize(s));
  });
}

int32_t net_graph_new_device(int64_t n, const uint32_t* d_src, const uint32_t* d_tgt,
                             const float* d_w32, const double* d_w64, int64_t m, int32_t directed,
                             GraphHandle** out, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    if (n < 0 || m < 0) throw Error("negative node or edge count");
    if ((uint64_t)n > 0xFFFFFFFFull)
      throw Error("node count (" + std::to_string(n) + ") exceeds the supported maximum");
    if ((uint64_t)m > 0xFFFFFFFFull / 2)
      throw Error("edge count (" + std::to_string(m) + ") exceeds the supported maximum");
    cudaStream_t s = knb::thread_stream();
    auto h = std::make_unique<GraphHandle>();
    knb::GraphHandleImpl& g = h->g;
    g.n = (uint32_t)n;
    g.m = (uint64_t)m;
    g.directed = directed != 0;
    g.weighted = d_w32 != nullptr || d_w64 != nullptr;
    KNB_CUDA(cudaGetDevice(&g.device));
    g.src.alloc(std::max<uint64_t>(g.m, 1));
    g.tgt.alloc(std::max<uint64_t>(g.m, 1));
    knb::DevBuf<unsigned long long> bad(1);
    if (m) {
      KNB_CUDA(cudaMemcpyAsync(g.src.get(), d_src, m * 4, cudaMemcpyDeviceToDevice, s));
      KNB_CUDA(cudaMemcpyAsync(g.tgt.get(), d_tgt, m * 4, cudaMemcpyDeviceToDevice, s));
      KNB_CUDA(cudaMemsetAsync(bad.get(), 0xFF, 8, s));
      check_u32_edges<<<knb::grid_for(m, 256), 256, 0, s>>>(g.src.get(), g.tgt.get(), m,
                                                            (uint64_t)n, bad.get());
      KNB_LAUNCH("check_u32_edges");
      uint64_t b = read_u64(bad.get(), s);
      if (b != NONE) throw Error("edge " + std::to_string(b / 2) + " refers to a node index out of range");
    }
    if (g.weighted) {
      g.w.alloc(std::max<uint64_t>(g.m, 1));
      if (m) {
        if (d_w64) {
          KNB_CUDA(cudaMemcpyAsync(g.w.get(), d_w64, m * 8, cudaMemcpyDeviceToDevice, s));
        } else {
          widen_weights<<<knb::grid_for(m, 256), 256, 0, s>>>(d_w32, m, g.w.get());
          KNB_LAUNCH("widen_weights");
        }
        KNB_CUDA(cudaMemsetAsync(bad.get(), 0xFF, 8, s));
        first_bad_weight<<<knb::grid_for(m, 256), 256, 0, s>>>(g.w.get(), m, 0, bad.get());
        KNB_LAUNCH("first_bad_weight");
        uint64_t e = read_u64(bad.get(), s);
        if (e != NONE)
          throw Error("edge " + std::to_string(e) + " has a missing, NaN, or infinite weight");
      }
    }
    finish_build(g, s);
    *out = h.release();
  });
}

// A graph handle over the edges frame_observed / frame_egos laid out.
static GraphHandle* frame_handle(knb::FrameEdges& fe, bool directed, bool weighted,
                                 int64_t* edge_rows, int64_t* edge_count, cudaStream_t s) {
  auto h = std::make_unique<GraphHandle>();
  knb::GraphHandleImpl& g = h->g;
  g.n = fe.n;
  g.m = fe.m;
  g.directed = directed;
  g.weighted = weighted;
  KNB_CUDA(cudaGetDevice(&g.device));
  g.src = std::move(fe.src);
  g.tgt = std::move(fe.tgt);
  if (weighted) g.w = std::move(fe.w);
  finish_build(g, s);
  if (edge_rows && fe.m) {
    std::vector<uint32_t> r(fe.m);
    KNB_CUDA(cudaMemcpyAsync(r.data(), fe.rows.get(), fe.m * 4, cudaMemcpyDeviceToHost, s));
    KNB_CUDA(cudaStreamSynchronize(s));
    for (uint64_t e = 0; e < fe.m; ++e) edge_rows[e] = r[e];
  }
  if (edge_count) *edge_count = (int64_t)fe.m;
  KNB_CUDA(cudaStreamSynchronize(s));
  return h.release();
}

int32_t net_frame_graph(int64_t n, const int64_t* src, const int64_t* tgt, const double* weights,
                        const uint8_t* missing, int64_t m, int32_t directed, GraphHandle** out,
                        int64_t* edge_rows, int64_t* edge_count, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    if (!out) throw Error("out is null");
    *out = nullptr;
    if (m > 0 && (!src || !tgt)) throw Error("an endpoint array is null");
    cudaStream_t s = knb::thread_stream();
    knb::FrameTable t{n, m, src, tgt, weights, missing};
    knb::FrameEdges fe;
    knb::frame_observed(t, &fe, s);
    *out = frame_handle(fe, directed != 0, weights != nullptr, edge_rows, edge_count, s);
  });
}

int32_t net_frame_egos(int64_t n, const int64_t* src, const int64_t* tgt, const double* weights,
                       const uint8_t* missing, int64_t m, int32_t directed,
                       const int64_t* node_ego, const int64_t* edge_ego, int64_t egos,
                       GraphHandle** out, int64_t* node_offsets, int64_t* node_ids,
                       int64_t* edge_rows, int64_t* edge_count, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    if (!out || !node_offsets) throw Error("out or node_offsets is null");
    *out = nullptr;
    if (m > 0 && (!src || !tgt)) throw Error("an endpoint array is null");
    if (n > 0 && !node_ego) throw Error("node_ego is null");
    cudaStream_t s = knb::thread_stream();
    knb::FrameTable t{n, m, src, tgt, weights, missing};
    knb::FrameEdges fe;
    knb::frame_egos(t, node_ego, edge_ego, egos, &fe, s);
    for (size_t k = 0; k < fe.node_offsets.size(); ++k) node_offsets[k] = fe.node_offsets[k];
    if (node_ids && fe.n) {
      std::vector<uint32_t> ids(fe.n);
      KNB_CUDA(cudaMemcpyAsync(ids.data(), fe.node_ids.get(), (size_t)fe.n * 4,
                               cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaStreamSynchronize(s));
      for (uint32_t i = 0; i < fe.n; ++i) node_ids[i] = ids[i];
    }
    *out = frame_handle(fe, directed != 0, weights != nullptr, edge_rows, edge_count, s);
  });
}

int32_t net_graph_edges(const GraphHandle* h, int64_t* src, int64_t* tgt, double* w, char* err,
                        size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    cudaStream_t s = knb::thread_stream();
    std::vector<uint32_t> a(g.m), b(g.m);
    if (g.m) {
      KNB_CUDA(cudaMemcpyAsync(a.data(), g.src.get(), g.m * 4, cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaMemcpyAsync(b.data(), g.tgt.get(), g.m * 4, cudaMemcpyDeviceToHost, s));
      if (w && g.weighted) KNB_CUDA(cudaMemcpyAsync(w, g.w.get(), g.m * 8, cudaMemcpyDeviceToHost, s));
    }
    KNB_CUDA(cudaStreamSynchronize(s));
    for (uint64_t e = 0; e < g.m; ++e) {
      if (src) src[e] = a[e];
      if (tgt) tgt[e] = b[e];
    }
  });
}

int32_t net_sweep_timing(int32_t phase, int64_t* launches, double* total_ms,
                         double* bytes_per_launch) {
  knb::SweepTiming t = knb::last_sweep_timing(phase);
  if (launches) *launches = t.launches;
  if (total_ms) *total_ms = t.ms;
  if (bytes_per_launch) *bytes_per_launch = t.bytes_per_launch;
  return 0;
}

void net_set_sweep_timing(int32_t on) { knb::set_sweep_timing(on != 0); }

int32_t net_set_tuning(int32_t key, double value) {
  knb::Tuning& t = knb::tuning();
  switch (key) {
    case 0:
      if (value != 0 && value != 4 && value != 8 && value != 16) return 1;
      t.ipt = (int)value;
      return 0;
    case 1:
      t.relabel = value != 0 ? 1 : 0;
      return 0;
    case 2:
      if (!(value >= 1)) return 1;
      t.switch_factor = value;
      return 0;
    case 3:
      if (!(value >= 0)) return 1;
      t.switch_floor = value;
      return 0;
    case 4:
      if (!(value >= 0 && value <= 12) || value != (int)value) return 1;
      t.variant = (int)value;
      return 0;
    case 5:
      if (!(value >= -1 && value <= 100)) return 1;
      t.carveout = (int)value;
      return 0;
    case 6:
      if (value != 0 && value != 128 && value != 256 && value != 512 && value != 1024) return 1;
      knb::set_ego_threads((int)value);
      return 0;
    case 7:
      if (!(value >= -1 && value <= 4294967295.0) || value != (double)(int64_t)value) return 1;
      t.hot_nodes = (int64_t)value;
      return 0;
    case 8:
      if (value != 0 && value != 1) return 1;
      t.persistent = (int)value;
      return 0;
    case 9:
      if (value != 0 && value != 1) return 1;
      t.refine = (int)value;
      return 0;
    case 10:
      if (!(value >= 0 && value <= 65535) || value != (int)value) return 1;
      t.long_row = (int)value;
      return 0;
    case 11:
      if (!(value >= -1 && value <= 1048576) || value != (int)value) return 1;
      t.smem_hot = (int64_t)value;
      return 0;
    case 12:
      if (value != 0 && value != 1) return 1;
      t.autotune = (int)value;
      return 0;
    case 13:
      if (!(value >= 0 && value <= 8) || value != (int)value) return 1;
      t.bulk_ctas = (int)value;
      return 0;
    case 14:
      if (!(value >= -1 && value <= 2147483647.0) || value != (double)(int64_t)value) return 1;
      t.bulk_skip_chunk = (int64_t)value;
      return 0;
    case 15:
      if (!(value >= 0 && value <= 4294967295.0) || value != (double)(int64_t)value) return 1;
      knb::set_ego_big_nodes((int64_t)value);
      return 0;
    case 16:
      if (value != 0 && value != 1 && value != 4 && value != 8) return 1;
      knb::set_ego_cluster((int)value);
      return 0;
    case 17:
      if (!(value >= 0 && value <= 4294967295.0) || value != (double)(int64_t)value) return 1;
      t.small_edges = (int64_t)value;
      return 0;
    default:
      return 1;
  }
}

int32_t net_projected_eigen(int64_t n, const double* a, double* values, double* vectors,
                            char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    if (n < 0 || n > 20) throw Error("the matrix order must be between 0 and 20");
    if (n == 0) return;
    if (!a || !values || !vectors) throw Error("a buffer is null");
    if (!knb::symmetric_eigen_device(a, (int)n, values, vectors, knb::thread_stream()))
      throw Error("the QL iteration did not converge");
  });
}

int32_t net_measure_gather(int32_t source, int64_t words, double* gathers_per_second, char* err,
                           size_t err_len) {
  return guard(err, err_len, [&] {
    if (!gathers_per_second) throw Error("gathers_per_second is null");
    if (source != 0 && source != 1 && source != 2 && source != 4 && source != 8)
      throw Error("gather source must be 0 (device array), 1 (shared memory) or 2, 4, 8 (cluster)");
    if (source == 0 && (words < 1024 || words > (int64_t(1) << 31)))
      throw Error("the array must hold between 1024 and 2^31 values");
    *gathers_per_second = knb::measure_gather_rate(source, (uint64_t)words, knb::thread_stream());
  });
}

// Row shards of one graph's PageRank (shard.cuh): the operator and the
// option checks of net_pagerank, then the split sweep.
static knb::Operator& shard_operator(knb::GraphHandleImpl& g, int32_t directed, int32_t weighted,
                                     int32_t loops, cudaStream_t s) {
  if (loops < 0 || loops > 2) throw Error("unknown self-loop weight code " + std::to_string(loops));
  const int which = knb::pagerank_rows(g, directed != 0);
  return g.op(which, weighted != 0, knb::pagerank_loop_factor(which, loops), s);
}

static cudaStream_t shard_stream(void* stream) {
  return stream ? static_cast<cudaStream_t>(stream) : cudaStream_t(0);
}

static knb::Shard& shard_of(const NetShard* sh) {
  if (!sh || !sh->s) throw Error("shard handle is null");
  return *sh->s;
}

int32_t net_shard_bounds(const GraphHandle* h, int32_t directed, int32_t weighted, int32_t loops,
                         int32_t parts, int64_t* bounds, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    if (!bounds) throw Error("bounds is null");
    cudaStream_t s = knb::thread_stream();
    knb::Operator& op = shard_operator(g, directed, weighted, loops, s);
    const std::vector<int64_t> b = knb::shard_bounds(op, parts, s);
    memcpy(bounds, b.data(), b.size() * 8);
  });
}

int32_t net_shard_new(const GraphHandle* h, double damping, int32_t directed, int32_t weighted,
                      const double* d_personalization, int32_t dangling, int32_t loops,
                      const int64_t* bounds, int32_t parts, int32_t rank, NetShard** shard,
                      int64_t* payload_len, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::GraphHandleImpl& g = handle(h);
    if (!shard || !bounds) throw Error("a buffer is null");
    *shard = nullptr;
    if (dangling != 0 && dangling != 1)
      throw Error("unknown dangling-node code " + std::to_string(dangling));
    if (loops < 0 || loops > 2) throw Error("unknown self-loop weight code " + std::to_string(loops));
    if (!(damping >= 0.0 && damping <= 1.0))
      throw Error("damping is " + fmt_g(damping) + "; it must be between 0 and 1");
    if (parts < 1 || parts > 1024) throw Error("the number of shards must be between 1 and 1024");
    cudaStream_t s = knb::thread_stream();
    if (weighted && g.n > 0) check_nonnegative(g, "PageRank", s);
    knb::Operator& op = shard_operator(g, directed, weighted, loops, s);
    knb::DevBuf<double> p;
    if (d_personalization && g.n > 0) {
      p.alloc(g.n);
      KNB_CUDA(cudaMemcpyAsync(p.get(), d_personalization, (size_t)g.n * 8,
                               cudaMemcpyDeviceToDevice, s));
      knb::normalize_personalization_device(p.get(), g.n, s);
    }
    const std::vector<int64_t> b(bounds, bounds + parts + 1);
    const bool uniform = !d_personalization || dangling == 1;
    auto out = std::make_unique<NetShard>();
    out->s = knb::shard_new(op, damping, p.get(), uniform, b, rank, s);
    if (payload_len) *payload_len = (int64_t)out->s->payload_len;
    *shard = out.release();
  });
}

int32_t net_shard_sweep(NetShard* shard, double* d_payload, void* stream, char* err,
                        size_t err_len) {
  return guard(err, err_len, [&] {
    knb::Shard& sh = shard_of(shard);
    if (!d_payload) throw Error("the payload buffer is null");
    knb::shard_sweep(sh, d_payload, shard_stream(stream));
  });
}

int32_t net_shard_restart(NetShard* shard, void* stream, char* err, size_t err_len) {
  return guard(err, err_len,
               [&] { knb::shard_restart(shard_of(shard), shard_stream(stream)); });
}

int32_t net_shard_finish(NetShard* shard, const double* d_gathered, double* change, void* stream,
                         char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::Shard& sh = shard_of(shard);
    if (!d_gathered || !change) throw Error("a buffer is null");
    *change = knb::shard_finish(sh, d_gathered, shard_stream(stream));
  });
}

int32_t net_shard_scores(const NetShard* shard, double* out, int32_t out_on_device, void* stream,
                         char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    knb::Shard& sh = shard_of(shard);
    if (sh.n == 0) return;
    if (!out) throw Error("the output buffer is null");
    knb::shard_scores(sh, out, out_on_device != 0, shard_stream(stream));
  });
}

void net_shard_free(NetShard* shard) { delete shard; }

int32_t net_device_sync(char* err, size_t err_len) {
  return guard(err, err_len, [&] { KNB_CUDA(cudaDeviceSynchronize()); });
}

}  // extern "C"
