// Many small graphs at once: PageRank on every block of a block-diagonal
// graph (ego networks, layers, subgraphs packed into one handle), in one
// persistent launch.
//
// Graphs are taken off queues largest first (so the last graphs to start are
// the small ones) and each runs the reference's iteration on its own
// (crates/engine/src/metrics/spectral.rs:247-280): z = x / out with the
// dangling mass `stuck`, y = A z, y = d (y + stuck jump) + (1 - d) p, the
// division by the total and the L1 change, every sum in a fixed order. Each
// graph therefore gets what a separate net_pagerank call on it returns, up to
// the association of sums. A large graph would keep one CTA busy long after
// the rest of the batch is done, so the launch runs in thread-block clusters:
// each cluster first splits the large graphs' rows over its CTAs, which add
// their sums through distributed shared memory, then every CTA takes small
// graphs alone. The vectors of the graph being solved stay in L2 (a graph's
// nodes are contiguous in the packed numbering). A single small graph's
// solve runs here too, as a batch of one.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <vector>

#include <cooperative_groups.h>

#include "ego.cuh"

namespace cg = cooperative_groups;

namespace knb {

struct EgoParams {
  double d;
  double tol;
  int32_t max_iter;
  int32_t jump_uniform;  // dangling nodes jump uniformly (1) or by p (0)
};

// Fixed-order CTA sums of K values at once (warp butterflies, then the warps
// in order): two CTA barriers for all K. sh holds 32 K doubles.
template <int K>
__device__ __forceinline__ void cta_sums(double (&v)[K], double* sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < K; ++j) v[j] = warp_sum(v[j]);
  __syncthreads();  // the previous sums' reads of sh are done
  if (lane == 0) {
#pragma unroll
    for (int j = 0; j < K; ++j) sh[32 * j + w] = v[j];
  }
  __syncthreads();
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double t = 0;
    for (int k = 0; k < nw; ++k) t += sh[32 * j + k];  // same order in every thread
    v[j] = t;
  }
}

// Sums over the rows of one graph split across the CTAs of a cluster: each
// CTA's fixed-order sums go to its slots, and every thread adds the slots in
// rank order through distributed shared memory, so all CTAs hold the same
// bits. The cluster barrier also publishes every global write made before
// it to the whole cluster (the z a product gathers from other CTAs' rows).
template <int C, int K>
__device__ __forceinline__ void cluster_sums(double (&v)[K], double* sh, double* slot,
                                             cg::cluster_group& cl) {
  cta_sums<K>(v, sh);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < K; ++j) slot[j] = v[j];
  }
  cl.sync();
#pragma unroll
  for (int j = 0; j < K; ++j) {
    double s = 0;
#pragma unroll
    for (int r = 0; r < C; ++r) s += cl.map_shared_rank(slot, (unsigned)r)[j];
    v[j] = s;
  }
}

// Fixed-order sums of K values over the rows of a graph: one CTA (C == 1)
// or a cluster. Slots (C > 1): two sets of 4 doubles of this CTA's shared
// memory, taken by turns, so a slot is written again only after every CTA
// has passed the next cluster barrier and so has read it.
template <int C, int K>
__device__ __forceinline__ void graph_sums(double (&v)[K], double* sh, double* slots, int turn) {
  if constexpr (C == 1) {
    (void)slots;
    (void)turn;
    cta_sums<K>(v, sh);
  } else {
    cg::cluster_group cl = cg::this_cluster();
    cluster_sums<C, K>(v, sh, slots + 4 * (turn & 1), cl);
  }
}

// One graph's iteration over rows [lo, hi) of nodes [g_lo, g_hi): the whole
// graph when C is 1 (one CTA), this CTA's share of it otherwise. The
// reference's steps (z = x / out with the dangling mass, y = A z, the
// update, the division by the total, the L1 change) with the next z and
// dangling mass formed in the same pass as the division and the change, so
// an iteration has two reductions (each a cluster barrier when C > 1).
template <int C>
__device__ void ego_solve(const OpView<double>& op, const double* __restrict__ outstr,
                          uint32_t g_lo, uint32_t g_hi, uint32_t lo, uint32_t hi,
                          const EgoParams& prm, const double* __restrict__ pers, double ps,
                          double* __restrict__ xa, double* __restrict__ xb,
                          double* __restrict__ zb, double* __restrict__ out, int32_t* it_out,
                          int32_t* done_out, double* change_out, double* sh, double* slots) {
  const uint32_t nk = g_hi - g_lo;
  const double inv_n = 1.0 / (double)nk;
  double* x = xa;
  double* y = xb;
  int turn = 0;
  // x = 1 / n; z = x / out; stuck = dangling mass
  double st[1] = {0.0};
  for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    x[i] = inv_n;
    const double o = outstr[i];
    if (o > 0.0) {
      zb[i] = inv_n / o;
    } else {
      zb[i] = 0.0;
      st[0] += inv_n;
    }
  }
  graph_sums<C, 1>(st, sh, slots, turn++);  // includes the barrier before z is read
  double stuck = st[0];
  int32_t it = 0, done = 0;
  double change = 0.0;
  while (it < prm.max_iter) {
    // y = d (A z + stuck jump) + (1 - d) p
    double tot[1] = {0.0};
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      // arcs in CSR order; four gathers in flight before their products
      // are added in that order
      double s = 0;
      uint32_t k = op.off[i];
      const uint32_t ke = op.off[i + 1];
      for (; k + 4 <= ke; k += 4) {
        double zk[4], wk[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          zk[u] = zb[op.cols[k + u]];
          wk[u] = op.vals ? op.vals[k + u] : 1.0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) s += wk[u] * zk[u];
      }
      for (; k < ke; ++k) {
        const double w = op.vals ? op.vals[k] : 1.0;
        s += w * zb[op.cols[k]];
      }
      const double p = pers ? pers[i] / ps : inv_n;
      const double jmp = prm.jump_uniform ? inv_n : p;
      const double v = prm.d * (s + stuck * jmp) + (1.0 - prm.d) * p;
      y[i] = v;
      tot[0] += v;
    }
    graph_sums<C, 1>(tot, sh, slots, turn++);  // every product has read z
    const double total = tot[0];
    // the division, the change, and the next z and dangling mass
    double cs[2] = {0.0, 0.0};
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
      const double v = y[i] / total;
      y[i] = v;
      cs[0] += fabs(v - x[i]);
      const double o = outstr[i];
      if (o > 0.0) {
        zb[i] = v / o;
      } else {
        zb[i] = 0.0;
        cs[1] += v;
      }
    }
    graph_sums<C, 2>(cs, sh, slots, turn++);  // publishes the next z
    change = cs[0];
    stuck = cs[1];
    double* t = x;
    x = y;
    y = t;
    ++it;
    if (change <= prm.tol) {  // the same bits in every CTA of a cluster
      done = 1;
      break;
    }
  }
  for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) out[i] = x[i];
  *it_out = it;
  *done_out = done;
  *change_out = change;
}

// The persistent launch. With clusters of C > 1 CTAs, each cluster first
// takes the large graphs (order[0, nbig), largest first) off queue[0], its
// CTAs splitting each graph's rows; once those are gone every CTA takes the
// other graphs (order[nbig, count)) off queue[1] alone. Cluster barriers
// are hardware barriers every CTA of the cluster executes the same number of
// times: the graph index comes from rank 0's shared memory, and every CTA
// stops a graph's iteration on the same bits.
template <int C>
__global__ void ego_pagerank(OpView<double> op, const double* __restrict__ outstr,
                             const uint32_t* __restrict__ node_off, const uint32_t* __restrict__ order,
                             uint32_t count, uint32_t nbig, unsigned int* __restrict__ queue,
                             EgoParams prm, const double* __restrict__ pers,
                             const double* __restrict__ psum, double* __restrict__ xa,
                             double* __restrict__ xb, double* __restrict__ zb,
                             double* __restrict__ out, int32_t* __restrict__ iters,
                             int32_t* __restrict__ status, double* __restrict__ changes) {
  __shared__ double sh[64];
  __shared__ double slots[8];
  __shared__ uint32_t g_sh;
  if constexpr (C > 1) {
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    for (;;) {
      if (rank == 0 && threadIdx.x == 0) g_sh = atomicAdd(queue, 1u);
      cl.sync();  // rank 0's pick is visible
      const uint32_t gi = *cl.map_shared_rank(&g_sh, 0u);
      cl.sync();  // every CTA has read it before rank 0 picks again or leaves
      if (gi >= nbig) break;
      const uint32_t graph = order[gi];
      const uint32_t g_lo = node_off[graph], g_hi = node_off[graph + 1];
      const uint32_t per = (g_hi - g_lo + C - 1) / C;
      const uint32_t lo = min(g_hi, g_lo + rank * per), hi = min(g_hi, lo + per);
      int32_t it = 0, done = 0;
      double ch = 0.0;
      ego_solve<C>(op, outstr, g_lo, g_hi, lo, hi, prm, pers, pers ? psum[graph] : 1.0, xa, xb,
                   zb, out, &it, &done, &ch, sh, slots);
      if (rank == 0 && threadIdx.x == 0) {
        iters[graph] = it;
        status[graph] = done ? 0 : 1;
        changes[graph] = ch;
      }
    }
  }
  for (;;) {
    if (threadIdx.x == 0) g_sh = atomicAdd(queue + 1, 1u);
    __syncthreads();
    const uint32_t gi = nbig + g_sh;
    __syncthreads();
    if (gi >= count) return;
    const uint32_t graph = order[gi];
    const uint32_t g_lo = node_off[graph], g_hi = node_off[graph + 1];
    if (g_hi == g_lo) {
      if (threadIdx.x == 0) {
        iters[graph] = 0;
        status[graph] = 0;
        changes[graph] = 0.0;
      }
      continue;
    }
    int32_t it = 0, done = 0;
    double ch = 0.0;
    ego_solve<1>(op, outstr, g_lo, g_hi, g_lo, g_hi, prm, pers, pers ? psum[graph] : 1.0, xa, xb,
                 zb, out, &it, &done, &ch, sh, slots);
    if (threadIdx.x == 0) {
      iters[graph] = it;
      status[graph] = done ? 0 : 1;
      changes[graph] = ch;
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

// Process-wide settings (net_set_tuning keys 6, 16, 15), read by solves that
// may run on other threads.
static std::atomic<int> g_ego_threads{0};  // 0: chosen per batch (tuned for large batches)
static std::atomic<int> g_ego_cluster{0};  // CTAs per cluster for the large graphs; 0: chosen
static std::atomic<int64_t> g_ego_big{0};  // nodes from which a graph is large; 0: automatic

void set_ego_threads(int t) { g_ego_threads = t; }
void set_ego_cluster(int c) { g_ego_cluster = c; }
void set_ego_big_nodes(int64_t v) { g_ego_big = v; }

// Clusters of C CTAs of `threads` that fit on the device at once (0 if none),
// per device and shape.
template <int C>
static int ego_clusters(int threads) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, int> cache;
  int dev = 0;
  KNB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find({dev, threads});
  if (it != cache.end()) return it->second;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(threads);
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  if (cudaOccupancyMaxActiveClusters(&clusters, (const void*)ego_pagerank<C>, &cfg) !=
      cudaSuccess) {
    cudaGetLastError();
    clusters = 0;
  }
  cache[{dev, threads}] = clusters;
  return clusters;
}

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
  std::vector<uint32_t> sizes;  // node counts of the graphs, largest first
  int tuned_threads = 0;       // this batch's choice (0: not chosen yet)
  int tuned_cluster = 0;
  int threads = 0;             // of the instantiated launch
  int cluster = 1;             // CTAs per cluster of the instantiated launch
  uint32_t nbig = 0;           // graphs it gives to clusters
  DevBuf<uint32_t> doff, dorder;
  DevBuf<double> dpers, dpsum, xa, xb, zb, dout;
  DevBuf<int32_t> iters, status;
  DevBuf<double> changes;
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
    P.tuned_threads = 0;
    P.tuned_cluster = 0;
    P.sizes.resize(count);
    for (uint32_t k = 0; k < count; ++k) P.sizes[k] = hoff[order[k] + 1] - hoff[order[k]];
    P.xa.alloc(n);
    P.xb.alloc(n);
    P.zb.alloc(n);
    P.dout.alloc(n);
    P.iters.alloc(count);
    P.status.alloc(count);
    P.changes.alloc(count);
    P.queue.alloc(2);
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
  // The launch: with clusters of C > 1 CTAs the graphs of at least `big`
  // nodes (by default max(4096, n / CTAs of the grid), so no graph holds
  // much more than a CTA's share of the batch) are each split over a
  // cluster; the others go one per CTA. Returns the graphs given to clusters.
  auto big_count = [&](uint64_t ctas) {
    const int64_t pin_big = g_ego_big.load();
    const uint64_t big = pin_big > 0 ? (uint64_t)pin_big
                                       : std::max<uint64_t>(4096, (uint64_t)n / std::max<uint64_t>(ctas, 1));
    uint32_t nb = 0;
    while (nb < count && P.sizes[nb] >= big) ++nb;
    return nb;
  };
  auto launch = [&](int threads, int C, cudaStream_t st) -> uint32_t {
    KNB_CUDA(cudaMemsetAsync(P.queue.get(), 0, 8, st));
    const uint64_t fit = (uint64_t)sms * (2048 / threads);
    int clusters = 0;
    if (C == 4) clusters = ego_clusters<4>(threads);
    if (C == 8) clusters = ego_clusters<8>(threads);
    const uint32_t nbig = clusters > 0 ? big_count((uint64_t)clusters * C) : 0;
    if (nbig == 0) {
      const unsigned grid = (unsigned)std::min<uint64_t>(count, fit);
      ego_pagerank<1><<<grid, threads, 0, st>>>(
          op.view64(), op.colsum.get(), P.doff.get(), P.dorder.get(), count, 0u, P.queue.get(),
          prm, pers ? P.dpers.get() : nullptr, pers ? P.dpsum.get() : nullptr, P.xa.get(),
          P.xb.get(), P.zb.get(), P.dout.get(), P.iters.get(), P.status.get(), P.changes.get());
      KNB_LAUNCH("ego_pagerank");
      return 0;
    }
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(clusters * C));
    cfg.blockDim = dim3((unsigned)threads);
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    auto args = [&](auto fn) {
      KNB_CUDA(cudaLaunchKernelEx(&cfg, fn, op.view64(), (const double*)op.colsum.get(),
                                  (const uint32_t*)P.doff.get(), (const uint32_t*)P.dorder.get(),
                                  count, nbig, P.queue.get(), prm,
                                  (const double*)(pers ? P.dpers.get() : nullptr),
                                  (const double*)(pers ? P.dpsum.get() : nullptr), P.xa.get(),
                                  P.xb.get(), P.zb.get(), P.dout.get(), P.iters.get(),
                                  P.status.get(), P.changes.get()));
    };
    if (C == 4) args(ego_pagerank<4>);
    else args(ego_pagerank<8>);
    KNB_LAUNCH("ego_pagerank");
    return nbig;
  };
  if (!P.t0) {
    KNB_CUDA(cudaEventCreate(&P.t0));
    KNB_CUDA(cudaEventCreate(&P.t1));
  }
  // Threads per CTA and CTAs per cluster, unless pinned (tuning keys 6 and
  // 16): for a batch of at least 2^20 arcs, timed once per batch layout on
  // the batch itself; smaller batches, whose launch takes microseconds, take
  // clusters of 8 and 1024 threads when they have fewer graphs than the GPU
  // has SMs (a single graph: 0.54 ms for C1 against 0.77 ms at 256), else
  // 256. Results do not depend on the choice beyond the association of a
  // split graph's sums.
  const int pin_t = g_ego_threads.load(), pin_c = g_ego_cluster.load();
  if (P.tuned_threads == 0) {
    int pick_t = pin_t ? pin_t : ((int)count < sms ? 1024 : 256);
    int pick_c = pin_c ? pin_c : 8;
    if ((pin_t == 0 || pin_c == 0) && op.nnz >= (1u << 20)) {
      float best = 1e30f;
      for (int t : {128, 256, 512, 1024}) {
        if (pin_t != 0 && t != pin_t) continue;
        for (int c : {1, 4, 8}) {
          if (pin_c != 0 && c != pin_c) continue;
          KNB_CUDA(cudaEventRecord(P.t0, s));
          launch(t, c, s);
          KNB_CUDA(cudaEventRecord(P.t1, s));
          KNB_CUDA(cudaEventSynchronize(P.t1));
          float ms = 0;
          KNB_CUDA(cudaEventElapsedTime(&ms, P.t0, P.t1));
          if (ms < best) {
            best = ms;
            pick_t = t;
            pick_c = c;
          }
        }
      }
    }
    P.tuned_threads = pick_t;
    P.tuned_cluster = pick_c;
  }
  const int threads = pin_t ? pin_t : P.tuned_threads;
  const int cluster = pin_c ? pin_c : P.tuned_cluster;
  if (!P.exec || P.threads != threads || P.cluster != cluster || P.pers != pers ||
      !same_params(P.prm, prm)) {
    P.drop_graph();
    cudaStream_t cs;
    KNB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    KNB_CUDA(cudaStreamSynchronize(s));
    KNB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    P.nbig = launch(threads, cluster, cs);
    KNB_CUDA(cudaStreamEndCapture(cs, &P.graph));
    KNB_CUDA(cudaGraphInstantiate(&P.exec, P.graph, 0));
    KNB_CUDA(cudaStreamDestroy(cs));
    P.threads = threads;
    P.cluster = cluster;
    P.pers = pers;
    P.prm = prm;
    ++P.instantiations;
  }
  KNB_CUDA(cudaEventRecord(P.t0, s));
  KNB_CUDA(cudaGraphLaunch(P.exec, s));
  KNB_CUDA(cudaEventRecord(P.t1, s));
  std::vector<int32_t> hst(count), hit(count);
  double change0 = 0.0;
  KNB_CUDA(cudaMemcpyAsync(hst.data(), P.status.get(), (size_t)count * 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaMemcpyAsync(hit.data(), P.iters.get(), (size_t)count * 4, cudaMemcpyDeviceToHost, s));
  if (count == 1)
    KNB_CUDA(cudaMemcpyAsync(&change0, P.changes.get(), 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  float ms = 0;
  KNB_CUDA(cudaEventElapsedTime(&ms, P.t0, P.t1));
  for (uint32_t k = 0; k < count; ++k)
    if (hst[k])
      throw Error("PageRank did not converge to tolerance " + std::to_string(in.tol) +
                  " within " + std::to_string(in.max_iter) + " iterations" +
                  (count > 1 ? " (graph " + std::to_string(k) + " of the batch)" : ""));
  if (in.out_on_device)
    KNB_CUDA(cudaMemcpyAsync(out, P.dout.get(), (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
  else
    KNB_CUDA(cudaMemcpyAsync(out, P.dout.get(), (size_t)n * 8, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  if (res) {
    res->seconds = ms * 1e-3;
    res->threads = threads;
    res->cluster = P.nbig ? cluster : 1;
    res->split_graphs = (int32_t)P.nbig;
    res->instantiations = P.instantiations;
    int64_t tot = 0, mx = 0;
    for (uint32_t k = 0; k < count; ++k) {
      tot += hit[k];
      mx = std::max<int64_t>(mx, hit[k]);
    }
    res->total_iterations = tot;
    res->change = change0;
    res->max_iterations = mx;
    if (in.iterations_out)
      for (uint32_t k = 0; k < count; ++k) in.iterations_out[k] = hit[k];
  }
}

}  // namespace knb
