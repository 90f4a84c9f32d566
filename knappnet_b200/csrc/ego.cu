// Many small graphs at once: PageRank on every block of a block-diagonal
// graph (ego networks, layers, subgraphs packed into one handle), in one
// persistent launch.
//
// Each CTA takes whole graphs off a queue, largest first (so the last graphs
// to start are the small ones), and runs the reference's iteration on that
// graph alone (crates/engine/src/metrics/spectral.rs:247-280): z = x / out
// with the dangling mass `stuck`, y = A z, y = d (y + stuck jump) + (1 - d) p,
// the division by the total and the L1 change, every step with CTA-wide
// reductions in a fixed order. Each graph therefore gets exactly what a
// separate net_pagerank call on it returns, up to the association of sums.
// The vectors of the graph being solved stay in L2 (a graph's nodes are
// contiguous in the packed numbering).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "ego.cuh"

namespace knb {

struct EgoParams {
  double d;
  double tol;
  int32_t max_iter;
  int32_t jump_uniform;  // dangling nodes jump uniformly (1) or by p (0)
};

// Fixed-order CTA sum (warp butterflies, then warp 0).
__device__ __forceinline__ double cta_sum(double v, double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = 0;
  for (int k = 0; k < nw; ++k) t += sh[k];  // same order in every thread
  return t;
}

__global__ void ego_pagerank(OpView<double> op, const double* __restrict__ outstr,
                             const uint32_t* __restrict__ node_off, const uint32_t* __restrict__ order,
                             uint32_t count, unsigned int* __restrict__ queue, EgoParams prm,
                             const double* __restrict__ pers, const double* __restrict__ psum,
                             double* __restrict__ xa, double* __restrict__ xb,
                             double* __restrict__ zb, double* __restrict__ out,
                             int32_t* __restrict__ iters, int32_t* __restrict__ status) {
  __shared__ double sh[32];
  __shared__ uint32_t g_sh;
  for (;;) {
    if (threadIdx.x == 0) g_sh = atomicAdd(queue, 1u);
    __syncthreads();
    const uint32_t gi = g_sh;
    __syncthreads();
    if (gi >= count) return;
    const uint32_t graph = order[gi];
    const uint32_t lo = node_off[graph], hi = node_off[graph + 1];
    const uint32_t nk = hi - lo;
    if (nk == 0) {
      if (threadIdx.x == 0) {
        iters[graph] = 0;
        status[graph] = 0;
      }
      continue;
    }
    const double inv_n = 1.0 / (double)nk;
    const double ps = pers ? psum[graph] : 1.0;
    double* x = xa;
    double* y = xb;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) x[i] = inv_n;
    __syncthreads();
    int32_t it = 0, done = 0;
    while (it < prm.max_iter) {
      // z = x / out; stuck = dangling mass
      double stuck = 0;
      for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const double o = outstr[i];
        if (o > 0.0) {
          zb[i] = x[i] / o;
        } else {
          zb[i] = 0.0;
          stuck += x[i];
        }
      }
      stuck = cta_sum(stuck, sh);  // includes the barrier before z is read
      // y = d (A z + stuck jump) + (1 - d) p
      double total = 0;
      for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        double s = 0;
        for (uint32_t k = op.off[i]; k < op.off[i + 1]; ++k) {
          const double w = op.vals ? op.vals[k] : 1.0;
          s += w * zb[op.cols[k]];
        }
        const double p = pers ? pers[i] / ps : inv_n;
        const double jmp = prm.jump_uniform ? inv_n : p;
        const double v = prm.d * (s + stuck * jmp) + (1.0 - prm.d) * p;
        y[i] = v;
        total += v;
      }
      total = cta_sum(total, sh);
      double change = 0;
      for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const double v = y[i] / total;
        y[i] = v;
        change += fabs(v - x[i]);
      }
      change = cta_sum(change, sh);
      double* t = x;
      x = y;
      y = t;
      ++it;
      if (change <= prm.tol) {
        done = 1;
        break;
      }
    }
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) out[i] = x[i];
    if (threadIdx.x == 0) {
      iters[graph] = it;
      status[graph] = done ? 0 : 1;
    }
    __syncthreads();
  }
}

// Edges must stay inside their graph: the first crossing edge, if any.
__global__ void ego_check_blocks(const uint32_t* __restrict__ src, const uint32_t* __restrict__ tgt,
                                 uint64_t m, const uint32_t* __restrict__ node_off, uint32_t count,
                                 unsigned long long* __restrict__ bad) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = src[e], b = tgt[e];
    // graph of a: largest k with node_off[k] <= a
    uint32_t lo = 0, hi = count;
    while (hi - lo > 1) {
      uint32_t mid = (lo + hi) >> 1;
      if (node_off[mid] <= a) lo = mid; else hi = mid;
    }
    if (b < node_off[lo] || b >= node_off[lo + 1]) atomicMin(bad, (unsigned long long)e);
  }
}

static int g_ego_threads = 0;  // 0: tuned on first use (per process)

void set_ego_threads(int t) { g_ego_threads = t; }

// A packed batch kept per operator between calls: the graph offsets and the
// largest-first order, every buffer, and the launch (queue reset and kernel)
// instantiated as a CUDA graph, which later calls with the same offsets,
// parameters and threads replay instead of capturing it again. Teleport
// values are copied in on every call. A call with other offsets rebuilds
// the plan; solves on one operator take turns on its mutex.
struct EgoPlan : Workspace {
  std::mutex mu;
  std::vector<uint32_t> hoff;  // the batch the buffers are laid out for
  bool pers = false;
  EgoParams prm{};
  int threads = 0;             // of the instantiated launch
  DevBuf<uint32_t> doff, dorder;
  DevBuf<double> dpers, dpsum, xa, xb, zb, dout;
  DevBuf<int32_t> iters, status;
  DevBuf<unsigned int> queue;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t t0 = nullptr, t1 = nullptr;
  int instantiations = 0;
  ~EgoPlan() override {
    drop_graph();
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
  }
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
};

static bool same_params(const EgoParams& a, const EgoParams& b) {
  return a.d == b.d && a.tol == b.tol && a.max_iter == b.max_iter &&
         a.jump_uniform == b.jump_uniform;
}

void pagerank_graphs(GraphHandleImpl& g, const EgoInput& in, double* out, EgoResult* res,
                     cudaStream_t s) {
  const uint32_t n = g.n;
  const uint32_t count = in.count;
  // node offsets: nondecreasing, from 0 to n
  if (in.node_offsets[0] != 0 || (uint64_t)in.node_offsets[count] != n)
    throw Error("graph offsets must start at 0 and end at the node count");
  for (uint32_t k = 0; k < count; ++k)
    if (in.node_offsets[k + 1] < in.node_offsets[k])
      throw Error("graph offsets must be nondecreasing");
  std::vector<uint32_t> hoff(count + 1);
  for (uint32_t k = 0; k <= count; ++k) hoff[k] = (uint32_t)in.node_offsets[k];
  // personalization: per-graph sums (host, in node order within each graph)
  std::vector<double> ps;
  if (in.personalization) {
    ps.assign(count, 0.0);
    for (uint32_t k = 0; k < count; ++k) {
      double t = 0;
      for (uint32_t i = hoff[k]; i < hoff[k + 1]; ++i) {
        double v = in.personalization[i];
        if (!std::isfinite(v) || v < 0.0)
          throw Error("the personalization vector must hold finite, nonnegative values");
        t += v;
      }
      if (hoff[k + 1] > hoff[k] && !(t > 0.0))
        throw Error("the personalization vector must have a positive sum");
      ps[k] = t;
    }
  }
  const int which = (g.directed && in.directed) ? 1 : (g.directed ? 2 : 0);
  const double lfac = in.loops == 2 ? 0.0 : (which == 1 ? 1.0 : (in.loops == 0 ? 2.0 : 1.0));
  Operator& op = g.op(which, in.weighted, lfac, s);
  EgoPlan* pp = nullptr;
  {
    std::lock_guard<std::mutex> lock(op.mu);
    if (!op.ego_ws) op.ego_ws = std::make_unique<EgoPlan>();
    pp = static_cast<EgoPlan*>(op.ego_ws.get());
  }
  EgoPlan& P = *pp;
  std::lock_guard<std::mutex> plan_lock(P.mu);
  const bool pers = in.personalization != nullptr;
  if (P.hoff != hoff) {
    // a new batch: check that no edge joins two graphs, order, buffers
    P.drop_graph();
    P.hoff.clear();
    P.doff.alloc(count + 1);
    P.dorder.alloc(std::max<uint32_t>(count, 1));
    KNB_CUDA(cudaMemcpyAsync(P.doff.get(), hoff.data(), (count + 1) * 4, cudaMemcpyHostToDevice, s));
    if (g.m) {
      DevBuf<unsigned long long> bad(1);
      KNB_CUDA(cudaMemsetAsync(bad.get(), 0xFF, 8, s));
      ego_check_blocks<<<grid_for(g.m, 256), 256, 0, s>>>(g.src.get(), g.tgt.get(), g.m,
                                                          P.doff.get(), count, bad.get());
      KNB_LAUNCH("ego_check_blocks");
      unsigned long long hb = 0;
      KNB_CUDA(cudaMemcpyAsync(&hb, bad.get(), 8, cudaMemcpyDeviceToHost, s));
      KNB_CUDA(cudaStreamSynchronize(s));
      if (hb != ~0ull)
        throw Error("edge " + std::to_string(hb) + " joins two different graphs of the batch");
    }
    // largest graphs first
    std::vector<uint32_t> order(count);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
      return hoff[a + 1] - hoff[a] > hoff[b + 1] - hoff[b];
    });
    KNB_CUDA(cudaMemcpyAsync(P.dorder.get(), order.data(), (size_t)count * 4,
                             cudaMemcpyHostToDevice, s));
    P.xa.alloc(n);
    P.xb.alloc(n);
    P.zb.alloc(n);
    P.dout.alloc(n);
    P.iters.alloc(count);
    P.status.alloc(count);
    P.queue.alloc(1);
    P.dpers.release();
    P.dpsum.release();
    KNB_CUDA(cudaStreamSynchronize(s));
    P.hoff = hoff;
  }
  if (pers && !P.dpers.get()) {
    P.dpers.alloc(n);
    P.dpsum.alloc(count);
  }
  if (pers) {
    KNB_CUDA(cudaMemcpyAsync(P.dpers.get(), in.personalization, (size_t)n * 8,
                             cudaMemcpyHostToDevice, s));
    KNB_CUDA(cudaMemcpyAsync(P.dpsum.get(), ps.data(), (size_t)count * 8, cudaMemcpyHostToDevice, s));
  }
  const EgoParams prm{in.damping, in.tol, (int32_t)std::min<int64_t>(in.max_iter, INT32_MAX),
                      in.dangling == 1 ? 1 : 0};
  int dev = 0, sms = 148;
  KNB_CUDA(cudaGetDevice(&dev));
  KNB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  auto launch = [&](int threads, cudaStream_t st) {
    KNB_CUDA(cudaMemsetAsync(P.queue.get(), 0, 4, st));
    const unsigned grid = (unsigned)std::min<uint64_t>(count, (uint64_t)sms * (2048 / threads));
    ego_pagerank<<<grid, threads, 0, st>>>(op.view64(), op.colsum.get(), P.doff.get(),
                                           P.dorder.get(), count, P.queue.get(), prm,
                                           pers ? P.dpers.get() : nullptr,
                                           pers ? P.dpsum.get() : nullptr, P.xa.get(), P.xb.get(),
                                           P.zb.get(), P.dout.get(), P.iters.get(),
                                           P.status.get());
    KNB_LAUNCH("ego_pagerank");
  };
  if (!P.t0) {
    KNB_CUDA(cudaEventCreate(&P.t0));
    KNB_CUDA(cudaEventCreate(&P.t1));
  }
  // Threads per CTA: tuned once per process by timing each candidate on
  // this batch (the results do not depend on the choice).
  if (g_ego_threads == 0) {
    float best = 1e30f;
    int pick = 256;
    for (int t : {128, 256, 512, 1024}) {
      KNB_CUDA(cudaEventRecord(P.t0, s));
      launch(t, s);
      KNB_CUDA(cudaEventRecord(P.t1, s));
      KNB_CUDA(cudaEventSynchronize(P.t1));
      float ms = 0;
      KNB_CUDA(cudaEventElapsedTime(&ms, P.t0, P.t1));
      if (ms < best) {
        best = ms;
        pick = t;
      }
    }
    g_ego_threads = pick;
  }
  const int threads = g_ego_threads;
  if (!P.exec || P.threads != threads || P.pers != pers || !same_params(P.prm, prm)) {
    P.drop_graph();
    cudaStream_t cs;
    KNB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    KNB_CUDA(cudaStreamSynchronize(s));
    KNB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    launch(threads, cs);
    KNB_CUDA(cudaStreamEndCapture(cs, &P.graph));
    KNB_CUDA(cudaGraphInstantiate(&P.exec, P.graph, 0));
    KNB_CUDA(cudaStreamDestroy(cs));
    P.threads = threads;
    P.pers = pers;
    P.prm = prm;
    ++P.instantiations;
  }
  KNB_CUDA(cudaEventRecord(P.t0, s));
  KNB_CUDA(cudaGraphLaunch(P.exec, s));
  KNB_CUDA(cudaEventRecord(P.t1, s));
  std::vector<int32_t> hst(count), hit(count);
  KNB_CUDA(cudaMemcpyAsync(hst.data(), P.status.get(), (size_t)count * 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaMemcpyAsync(hit.data(), P.iters.get(), (size_t)count * 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  KNB_CUDA(cudaEventElapsedTime(&ms, P.t0, P.t1));
  for (uint32_t k = 0; k < count; ++k)
    if (hst[k])
      throw Error("PageRank did not converge to tolerance " + std::to_string(in.tol) +
                  " within " + std::to_string(in.max_iter) + " iterations (graph " +
                  std::to_string(k) + " of the batch)");
  if (in.out_on_device)
    KNB_CUDA(cudaMemcpyAsync(out, P.dout.get(), (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
  else
    KNB_CUDA(cudaMemcpyAsync(out, P.dout.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  if (res) {
    res->seconds = ms * 1e-3;
    res->threads = threads;
    res->instantiations = P.instantiations;
    int64_t tot = 0, mx = 0;
    for (uint32_t k = 0; k < count; ++k) {
      tot += hit[k];
      mx = std::max<int64_t>(mx, hit[k]);
    }
    res->total_iterations = tot;
    res->max_iterations = mx;
    if (in.iterations_out)
      for (uint32_t k = 0; k < count; ++k) in.iterations_out[k] = hit[k];
  }
}

}  // namespace knb
