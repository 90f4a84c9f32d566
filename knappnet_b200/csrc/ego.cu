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
#include <cstring>
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
  DevBuf<uint32_t> doff(count + 1), dorder(std::max<uint32_t>(count, 1));
  KNB_CUDA(cudaMemcpyAsync(doff.get(), hoff.data(), (count + 1) * 4, cudaMemcpyHostToDevice, s));
  if (g.m) {
    DevBuf<unsigned long long> bad(1);
    KNB_CUDA(cudaMemsetAsync(bad.get(), 0xFF, 8, s));
    ego_check_blocks<<<grid_for(g.m, 256), 256, 0, s>>>(g.src.get(), g.tgt.get(), g.m, doff.get(),
                                                        count, bad.get());
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
  KNB_CUDA(cudaMemcpyAsync(dorder.get(), order.data(), (size_t)count * 4, cudaMemcpyHostToDevice, s));

  const int which = (g.directed && in.directed) ? 1 : (g.directed ? 2 : 0);
  const double lfac = in.loops == 2 ? 0.0 : (which == 1 ? 1.0 : (in.loops == 0 ? 2.0 : 1.0));
  Operator& op = g.op(which, in.weighted, lfac, s);

  // personalization: per-graph sums (host, in node order within each graph)
  DevBuf<double> dpers, dpsum;
  if (in.personalization) {
    std::vector<double> ps(count, 0.0);
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
    dpers.alloc(n);
    dpsum.alloc(count);
    KNB_CUDA(cudaMemcpyAsync(dpers.get(), in.personalization, (size_t)n * 8, cudaMemcpyHostToDevice, s));
    KNB_CUDA(cudaMemcpyAsync(dpsum.get(), ps.data(), (size_t)count * 8, cudaMemcpyHostToDevice, s));
  }
  DevBuf<double> xa(n), xb(n), zb(n), dout(n);
  DevBuf<int32_t> iters(count), status(count);
  DevBuf<unsigned int> queue(1);
  EgoParams prm{in.damping, in.tol, (int32_t)std::min<int64_t>(in.max_iter, INT32_MAX),
                in.dangling == 1 ? 1 : 0};
  int dev = 0, sms = 148;
  KNB_CUDA(cudaGetDevice(&dev));
  KNB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));

  auto launch = [&](int threads) {
    KNB_CUDA(cudaMemsetAsync(queue.get(), 0, 4, s));
    const unsigned grid = (unsigned)std::min<uint64_t>(count, (uint64_t)sms * (2048 / threads));
    ego_pagerank<<<grid, threads, 0, s>>>(op.view64(), op.colsum.get(), doff.get(), dorder.get(),
                                          count, queue.get(), prm, dpers.get(), dpsum.get(),
                                          xa.get(), xb.get(), zb.get(), dout.get(), iters.get(),
                                          status.get());
    KNB_LAUNCH("ego_pagerank");
  };
  // Threads per CTA: tuned once per process by timing each candidate on
  // this batch (the results do not depend on the choice).
  if (g_ego_threads == 0) {
    float best = 1e30f;
    int pick = 256;
    cudaEvent_t a, b;
    KNB_CUDA(cudaEventCreate(&a));
    KNB_CUDA(cudaEventCreate(&b));
    for (int t : {128, 256, 512, 1024}) {
      KNB_CUDA(cudaEventRecord(a, s));
      launch(t);
      KNB_CUDA(cudaEventRecord(b, s));
      KNB_CUDA(cudaEventSynchronize(b));
      float ms = 0;
      KNB_CUDA(cudaEventElapsedTime(&ms, a, b));
      if (ms < best) {
        best = ms;
        pick = t;
      }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    g_ego_threads = pick;
  }
  const int threads = g_ego_threads;

  // The launch sequence (queue reset + kernel) as a CUDA graph.
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  cudaStream_t cs;
  KNB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  KNB_CUDA(cudaStreamSynchronize(s));
  KNB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  {
    cudaStream_t keep = s;
    s = cs;
    launch(threads);
    s = keep;
  }
  KNB_CUDA(cudaStreamEndCapture(cs, &graph));
  KNB_CUDA(cudaGraphInstantiate(&exec, graph, 0));
  cudaEvent_t t0, t1;
  KNB_CUDA(cudaEventCreate(&t0));
  KNB_CUDA(cudaEventCreate(&t1));
  KNB_CUDA(cudaEventRecord(t0, cs));
  KNB_CUDA(cudaGraphLaunch(exec, cs));
  KNB_CUDA(cudaEventRecord(t1, cs));
  KNB_CUDA(cudaStreamSynchronize(cs));
  float ms = 0;
  KNB_CUDA(cudaEventElapsedTime(&ms, t0, t1));
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  cudaStreamDestroy(cs);

  std::vector<int32_t> hst(count), hit(count);
  KNB_CUDA(cudaMemcpyAsync(hst.data(), status.get(), (size_t)count * 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaMemcpyAsync(hit.data(), iters.get(), (size_t)count * 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  for (uint32_t k = 0; k < count; ++k)
    if (hst[k])
      throw Error("PageRank did not converge to tolerance " + std::to_string(in.tol) +
                  " within " + std::to_string(in.max_iter) + " iterations (graph " +
                  std::to_string(k) + " of the batch)");
  if (in.out_on_device)
    KNB_CUDA(cudaMemcpyAsync(out, dout.get(), (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
  else
    KNB_CUDA(cudaMemcpyAsync(out, dout.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  if (res) {
    res->seconds = ms * 1e-3;
    res->threads = threads;
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
