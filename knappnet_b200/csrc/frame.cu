// Graphs from a frame's resolved edge table on the device (reference:
// crates/engine/src/frame/build.rs:106-121 graph_of, :153-194 subgraph,
// :220-238 ego_subgraph). The reference builds each ego's subgraph as its own
// graph, one call at a time; here all egos are cut out in one pass and packed
// back to back into one graph, the input net_pagerank_graphs solves in one
// launch. Row and node orders are the reference's: a subgraph keeps its nodes
// ascending and its rows in table order, and a stable sort by ego label
// preserves both.
#include <algorithm>
#include <cmath>
#include <string>

#include "frame.cuh"
#include "graph.cuh"

namespace knb {

constexpr unsigned long long FRAME_NONE = ~0ull;

// The first observed row with an endpoint outside [0, n) and the first with
// a weight that is not finite; endpoints as 32-bit node indices.
__global__ void frame_check(const int64_t* __restrict__ s64, const int64_t* __restrict__ t64,
                            const double* __restrict__ w, const uint8_t* __restrict__ missing,
                            uint64_t m, uint64_t n, uint32_t* __restrict__ s32,
                            uint32_t* __restrict__ t32, unsigned long long* __restrict__ bad_end,
                            unsigned long long* __restrict__ bad_w) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const bool seen = missing == nullptr || missing[e] == 0;
    const int64_t a = s64[e], b = t64[e];
    const bool ok = a >= 0 && b >= 0 && (uint64_t)a < n && (uint64_t)b < n;
    if (seen && !ok) atomicMin(bad_end, (unsigned long long)e);
    if (seen && w && !isfinite(w[e])) atomicMin(bad_w, (unsigned long long)e);
    s32[e] = ok ? (uint32_t)a : 0u;
    t32[e] = ok ? (uint32_t)b : 0u;
  }
}

__global__ void frame_seen_flags(const uint8_t* __restrict__ missing, uint64_t m,
                                 uint32_t* __restrict__ flag) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x)
    flag[e] = (missing == nullptr || missing[e] == 0) ? 1u : 0u;
}

// Observed rows to their place (pos: exclusive scan of the flags).
__global__ void frame_compact(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos,
                              const uint32_t* __restrict__ s32, const uint32_t* __restrict__ t32,
                              const double* __restrict__ w, uint64_t m, uint32_t* __restrict__ so,
                              uint32_t* __restrict__ to, double* __restrict__ wo,
                              uint32_t* __restrict__ rows) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    if (!flag[e]) continue;
    const uint32_t q = pos[e];
    so[q] = s32[e];
    to[q] = t32[e];
    if (w) wo[q] = w[e];
    rows[q] = (uint32_t)e;
  }
}

// Sort keys: (ego, index) for members, all ones for the rest (sorted last).
__global__ void frame_node_keys(const int32_t* __restrict__ ego, uint32_t n,
                                unsigned long long* __restrict__ keys, uint32_t* __restrict__ ids,
                                uint32_t* __restrict__ count) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int32_t k = ego[i];
    keys[i] = k >= 0 ? ((unsigned long long)k << 32 | i) : FRAME_NONE;
    ids[i] = i;
    if (k >= 0) atomicAdd(count + k, 1u);
  }
}

__global__ void frame_node_index(const uint32_t* __restrict__ ids, uint32_t kept,
                                 uint32_t* __restrict__ newid) {
  for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < kept; p += gridDim.x * blockDim.x)
    newid[ids[p]] = p;
}

// A row belongs to ego k when it is observed, labelled k, and both its
// endpoints are members of ego k (subgraph drops rows with a dropped end).
// Without edge labels a row takes its source's ego, as the reference's
// resolved ego codes do (crates/engine/src/frame/validate.rs:115-117).
__global__ void frame_edge_keys(const int32_t* __restrict__ node_ego,
                                const int32_t* __restrict__ edge_ego,
                                const uint8_t* __restrict__ missing,
                                const uint32_t* __restrict__ s32, const uint32_t* __restrict__ t32,
                                uint64_t m, unsigned long long* __restrict__ keys,
                                uint32_t* __restrict__ ids, unsigned int* __restrict__ kept) {
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e < m;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const int32_t k = edge_ego ? edge_ego[e] : node_ego[s32[e]];
    const bool in = k >= 0 && (missing == nullptr || missing[e] == 0) &&
                    node_ego[s32[e]] == k && node_ego[t32[e]] == k;
    keys[e] = in ? ((unsigned long long)k << 32 | e) : FRAME_NONE;
    ids[e] = (uint32_t)e;
    if (in) atomicAdd(kept, 1u);
  }
}

__global__ void frame_pack_edges(const uint32_t* __restrict__ order, uint64_t kept,
                                 const uint32_t* __restrict__ newid,
                                 const uint32_t* __restrict__ s32, const uint32_t* __restrict__ t32,
                                 const double* __restrict__ w, uint32_t* __restrict__ so,
                                 uint32_t* __restrict__ to, double* __restrict__ wo,
                                 uint32_t* __restrict__ rows) {
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < kept;
       q += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t e = order[q];
    so[q] = newid[s32[e]];
    to[q] = newid[t32[e]];
    if (w) wo[q] = w[e];
    rows[q] = e;
  }
}

namespace {

// Uploads the table, checks it, and leaves 32-bit endpoints on the device.
struct Uploaded {
  DevBuf<uint32_t> s32, t32;
  DevBuf<double> w;
  DevBuf<uint8_t> missing;
};

void upload(const FrameTable& t, Uploaded* u, cudaStream_t s) {
  if (t.n < 0 || t.m < 0) throw Error("negative node or edge count");
  if ((uint64_t)t.n > 0xFFFFFFFFull)
    throw Error("node count (" + std::to_string(t.n) + ") exceeds the supported maximum");
  if ((uint64_t)t.m > 0xFFFFFFFFull / 2)
    throw Error("edge count (" + std::to_string(t.m) + ") exceeds the supported maximum");
  const uint64_t m = (uint64_t)t.m;
  const size_t mm = std::max<uint64_t>(m, 1);
  u->s32.alloc(mm);
  u->t32.alloc(mm);
  if (t.weights) u->w.alloc(mm);
  if (t.missing) u->missing.alloc(mm);
  if (m == 0) return;
  DevBuf<int64_t> s64(m), t64(m);
  DevBuf<unsigned long long> bad(2);
  KNB_CUDA(cudaMemcpyAsync(s64.get(), t.src, m * 8, cudaMemcpyHostToDevice, s));
  KNB_CUDA(cudaMemcpyAsync(t64.get(), t.tgt, m * 8, cudaMemcpyHostToDevice, s));
  if (t.weights) KNB_CUDA(cudaMemcpyAsync(u->w.get(), t.weights, m * 8, cudaMemcpyHostToDevice, s));
  if (t.missing)
    KNB_CUDA(cudaMemcpyAsync(u->missing.get(), t.missing, m, cudaMemcpyHostToDevice, s));
  KNB_CUDA(cudaMemsetAsync(bad.get(), 0xFF, 16, s));
  frame_check<<<grid_for(m, 256), 256, 0, s>>>(s64.get(), t64.get(), u->w.get(),
                                                u->missing.get(), m, (uint64_t)t.n, u->s32.get(),
                                                u->t32.get(), bad.get(), bad.get() + 1);
  KNB_LAUNCH("frame_check");
  unsigned long long hb[2];
  KNB_CUDA(cudaMemcpyAsync(hb, bad.get(), 16, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  // Graph::from_edges (crates/engine/src/graph.rs:162-192) checks every
  // weight before any endpoint and numbers edges among the rows it was given:
  // here the observed rows.
  auto edge_of = [&](uint64_t row) {
    uint64_t k = row;
    if (t.missing)
      for (uint64_t e = 0; e < row; ++e) k -= t.missing[e] != 0;
    return std::to_string(k);
  };
  if (hb[1] != FRAME_NONE)
    throw Error("edge " + edge_of(hb[1]) + " has a missing, NaN, or infinite weight");
  if (hb[0] != FRAME_NONE) {
    const uint64_t e = hb[0];
    const int64_t a = t.src[e], b = t.tgt[e];
    const int64_t bad = (a < 0 || a >= t.n) ? a : b;
    throw Error("edge " + edge_of(e) + " refers to node index " + std::to_string(bad) +
                ", but valid indices are 0.." + std::to_string(t.n));
  }
}

// Ego labels as 32-bit values, -1 for anything outside 0..egos-1.
DevBuf<int32_t> labels(const int64_t* v, uint64_t count, int64_t egos, cudaStream_t s) {
  std::vector<int32_t> h(count);
  for (uint64_t i = 0; i < count; ++i)
    h[i] = (v[i] >= 0 && v[i] < egos) ? (int32_t)v[i] : -1;
  DevBuf<int32_t> d(std::max<uint64_t>(count, 1));
  if (count)
    KNB_CUDA(cudaMemcpyAsync(d.get(), h.data(), count * 4, cudaMemcpyHostToDevice, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  return d;
}

}  // namespace

void frame_observed(const FrameTable& t, FrameEdges* out, cudaStream_t s) {
  Uploaded u;
  upload(t, &u, s);
  const uint64_t m = (uint64_t)t.m;
  out->n = (uint32_t)t.n;
  DevBuf<uint32_t> flag(m + 1), pos(m + 1);
  uint64_t kept = 0;
  if (m) {
    frame_seen_flags<<<grid_for(m, 256), 256, 0, s>>>(u.missing.get(), m, flag.get());
    KNB_LAUNCH("frame_seen_flags");
    kept = exclusive_scan<uint32_t>(flag.get(), pos.get(), m, s);
  }
  out->m = kept;
  const size_t km = std::max<uint64_t>(kept, 1);
  out->src.alloc(km);
  out->tgt.alloc(km);
  out->rows.alloc(km);
  if (t.weights) out->w.alloc(km);
  if (m) {
    frame_compact<<<grid_for(m, 256), 256, 0, s>>>(flag.get(), pos.get(), u.s32.get(),
                                                    u.t32.get(), u.w.get(), m, out->src.get(),
                                                    out->tgt.get(), out->w.get(), out->rows.get());
    KNB_LAUNCH("frame_compact");
  }
  KNB_CUDA(cudaStreamSynchronize(s));
}

void frame_egos(const FrameTable& t, const int64_t* node_ego, const int64_t* edge_ego,
                int64_t egos, FrameEdges* out, cudaStream_t s) {
  if (egos < 0 || egos > 0x7FFFFFFFll) throw Error("ego count out of range");
  Uploaded u;
  upload(t, &u, s);
  const uint32_t n = (uint32_t)t.n;
  const uint64_t m = (uint64_t)t.m;
  DevBuf<int32_t> nego = labels(node_ego, n, egos, s);
  DevBuf<int32_t> eego;
  if (edge_ego) eego = labels(edge_ego, m, egos, s);
  // members of every ego, ego by ego, ascending within each
  DevBuf<unsigned long long> nkeys(std::max<uint32_t>(n, 1));
  DevBuf<uint32_t> nids(std::max<uint32_t>(n, 1));
  DevBuf<uint32_t> count((size_t)egos + 1);
  KNB_CUDA(cudaMemsetAsync(count.get(), 0, ((size_t)egos + 1) * 4, s));
  if (n) {
    frame_node_keys<<<grid_for(n, 256), 256, 0, s>>>(nego.get(), n, nkeys.get(), nids.get(),
                                                      count.get());
    KNB_LAUNCH("frame_node_keys");
    radix_sort(reinterpret_cast<uint64_t*>(nkeys.get()), nids.get(), n, 64, s);
  }
  const uint32_t members = exclusive_scan<uint32_t>(count.get(), count.get(), (size_t)egos + 1, s);
  std::vector<uint32_t> hoff((size_t)egos + 1);
  KNB_CUDA(cudaMemcpyAsync(hoff.data(), count.get(), hoff.size() * 4, cudaMemcpyDeviceToHost, s));
  DevBuf<uint32_t> newid(std::max<uint32_t>(n, 1));
  if (members) {
    frame_node_index<<<grid_for(members, 256), 256, 0, s>>>(nids.get(), members, newid.get());
    KNB_LAUNCH("frame_node_index");
  }
  // rows of every ego, ego by ego, in row order within each
  DevBuf<unsigned long long> ekeys(std::max<uint64_t>(m, 1));
  DevBuf<uint32_t> eids(std::max<uint64_t>(m, 1));
  DevBuf<unsigned int> kept_d(1);
  KNB_CUDA(cudaMemsetAsync(kept_d.get(), 0, 4, s));
  if (m) {
    frame_edge_keys<<<grid_for(m, 256), 256, 0, s>>>(nego.get(), eego.get(), u.missing.get(),
                                                      u.s32.get(), u.t32.get(), m, ekeys.get(),
                                                      eids.get(), kept_d.get());
    KNB_LAUNCH("frame_edge_keys");
    radix_sort(reinterpret_cast<uint64_t*>(ekeys.get()), eids.get(), m, 64, s);
  }
  unsigned int kept = 0;
  KNB_CUDA(cudaMemcpyAsync(&kept, kept_d.get(), 4, cudaMemcpyDeviceToHost, s));
  KNB_CUDA(cudaStreamSynchronize(s));
  out->n = members;
  out->m = kept;
  out->node_offsets.assign(hoff.begin(), hoff.end());
  out->node_ids.alloc(std::max<uint32_t>(members, 1));
  if (members)
    KNB_CUDA(cudaMemcpyAsync(out->node_ids.get(), nids.get(), (size_t)members * 4,
                             cudaMemcpyDeviceToDevice, s));
  const size_t km = std::max<uint32_t>(kept, 1);
  out->src.alloc(km);
  out->tgt.alloc(km);
  out->rows.alloc(km);
  if (t.weights) out->w.alloc(km);
  if (kept) {
    frame_pack_edges<<<grid_for(kept, 256), 256, 0, s>>>(eids.get(), kept, newid.get(),
                                                          u.s32.get(), u.t32.get(), u.w.get(),
                                                          out->src.get(), out->tgt.get(),
                                                          out->w.get(), out->rows.get());
    KNB_LAUNCH("frame_pack_edges");
  }
  KNB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace knb
