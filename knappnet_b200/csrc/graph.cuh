// Device-resident graph handle and the operators built from it.
#pragma once

#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "common.cuh"
#include "slice.cuh"
#include "spmv.cuh"

namespace knb {

// One direction of adjacency in CSR layout on the device, as the reference's
// Csr (crates/engine/src/graph.rs:19-24): arcs of node v are
// tgt[off[v] .. off[v+1]], sorted by target, parallel arcs in input order.
// Offsets are 32-bit: the reference caps the edge count at u32::MAX / 2
// (graph.rs:175), so an undirected graph has fewer than 2^32 arcs.
struct DevCsr {
  uint32_t n = 0;
  uint64_t arcs = 0;
  DevBuf<uint32_t> off;   // n + 1
  DevBuf<uint32_t> tgt;   // arcs
  DevBuf<uint32_t> edge;  // arcs: the input edge each arc comes from
  DevBuf<double> w;       // arcs, weighted graphs only
};

// Merge-path partition of an operator for one tile width.
struct Partition {
  uint32_t tile = 0;         // merge items per tile
  uint32_t ntiles = 0;
  DevBuf<TileCoord> coords;  // ntiles + 1
  DevBuf<SplitRow> split;    // rows spanning <= SHORT_SPAN tiles first, then the rest
  uint32_t nsplit = 0;
  uint32_t nshort = 0;
};
constexpr uint32_t SHORT_SPAN = 16;

// An operator with its nodes renumbered by decreasing column count (how
// often a sweep gathers each node's value), ties by node: the values most
// gathered then sit together in a few MB, so their cache lines stay in L2 and
// L1 instead of being spread over the whole iterate. perm[k] is the node
// whose new number is k; iperm is its inverse. Rows keep their arc order with
// columns renamed, so row sums add the same terms in the same order.
struct Relabeled {
  DevBuf<uint32_t> perm, iperm, off, cols;
  DevBuf<double> vals64;
  DevBuf<float> vals32;
  DevBuf<double> inv_out64;
  DevBuf<float> inv_out32;
  std::map<uint32_t, std::unique_ptr<Partition>> parts;
};

// An operator in the sliced layout of slice.cuh: nodes renumbered by
// decreasing row length, ties by decreasing column count, then by node
// (perm[k] is the node whose new number is k, iperm its inverse). Each row's
// arcs are sorted by renamed column (parallel arcs keep their order); rows
// of at least `lw` arcs form a row-compressed part cut into pieces of
// `piece` arcs, the others slices of 32 rows stored arc-major. Row sums add
// the same terms as the reference's, in column order.
struct SlicedOp {
  uint32_t n = 0;
  uint64_t nnz = 0;
  uint32_t lw = 0;
  uint32_t n_long = 0;
  uint32_t long_arcs = 0;
  uint32_t piece = 0;
  uint32_t npieces = 0;
  uint32_t nslices = 0;
  uint64_t slice_elems = 0;  // arc-major elements, padding included
  DevBuf<uint32_t> perm, iperm;
  DevBuf<uint32_t> loff, lcols, prow;
  DevBuf<double> lvals64;
  DevBuf<float> lvals32;
  DevBuf<uint32_t> sbase, scols;
  DevBuf<uint16_t> slen;
  DevBuf<double> svals64;
  DevBuf<float> svals32;
  DevBuf<double> inv_out64;
  DevBuf<float> inv_out32;
  DevBuf<SplitRow> split;  // rows cut by piece boundaries (split_rows)
  uint32_t nsplit = 0;
  uint32_t nshort = 0;
  bool has_vals = false;
  SliceView<double> view64() const {
    return {n, n_long, long_arcs, piece, npieces, nslices, loff.get(), lcols.get(),
            has_vals ? lvals64.get() : nullptr, prow.get(), sbase.get(), slen.get(),
            scols.get(), has_vals ? svals64.get() : nullptr};
  }
  SliceView<float> view32() const {
    return {n, n_long, long_arcs, piece, npieces, nslices, loff.get(), lcols.get(),
            has_vals ? lvals32.get() : nullptr, prow.get(), sbase.get(), slen.get(),
            scols.get(), has_vals ? svals32.get() : nullptr};
  }
  template <class MT>
  SliceView<MT> view() const {
    if constexpr (sizeof(MT) == 8) return view64(); else return view32();
  }
};

// The PageRank sweep a tuner picked for an operator: kernel (tuning key 4
// codes), long-row threshold of the sliced layout, columns whose gathers
// allocate in L1 (in FP32 values), and its measured time per sweep.
struct SweepPick {
  int32_t variant = 0;
  int32_t long_row = 0;
  int32_t ipt = 0;
  int64_t hot = -1;
  double ms = 0;
};

// Per-operator scratch a solver keeps between calls (iterates, partials,
// events), so a call allocates nothing once warm.
struct Workspace {
  virtual ~Workspace() = default;
};

// The matrix a measure multiplies by: rows of one adjacency with arc values
// (weights or 1, self-loops times their diagonal factor), as SparseOp::from_rows
// (crates/engine/src/metrics/eigenvector.rs:512-547); plus the column sums
// (out-strength for PageRank's pull operator) and their reciprocals.
struct Operator {
  const DevCsr* rows = nullptr;
  uint32_t n = 0;
  uint64_t nnz = 0;
  bool has_vals = false;
  bool vals32_exact = false;  // every value is exactly representable in FP32
  DevBuf<double> vals64;
  DevBuf<float> vals32;
  DevBuf<double> colsum;      // column sums (out-strength of the pull operator)
  DevBuf<double> inv_out64;   // 1 / colsum, 0 where colsum == 0 (dangling)
  DevBuf<float> inv_out32;
  uint32_t n_dangling = 0;
  std::map<uint32_t, std::unique_ptr<Partition>> parts;
  std::mutex mu;  // guards parts and relabel
  const DevCsr* trans = nullptr;  // adjacency whose row lengths are this operator's column counts
  std::unique_ptr<Relabeled> relabel;
  std::map<std::pair<uint32_t, uint32_t>, std::unique_ptr<SlicedOp>> sliced_ops;  // (lw, pieces)
  std::map<int, SweepPick> pr_pick;  // PageRank's tuned sweep per precision class (pagerank.cu), under mu
  std::unique_ptr<Workspace> pr_ws;  // PageRank's (pagerank.cu), created on first use
  std::unique_ptr<Workspace> eig_ws;  // eigenvector centrality's (eigen.cu), created on first use
  std::unique_ptr<Workspace> hits_ws;  // hubs and authorities' (eigen.cu), created on first use
  std::unique_ptr<Workspace> series_ws;  // the Katz / Bonacich attenuation check's (katz.cu)
  std::map<int, int> batch_u;  // batched PageRank's tuned arcs in flight (batch.cu), under mu
  std::unique_ptr<Workspace> batch_ws;  // batched PageRank's plan and buffers (batch.cu)
  std::unique_ptr<Workspace> ego_ws;  // packed-graph PageRank's plan and launch graph (ego.cu)

  const Relabeled& relabeled(cudaStream_t s);
  const Partition& relabeled_partition(uint32_t tile_items, cudaStream_t s);
  // The sliced layout with long rows of at least lw (<= 65535) arcs cut into
  // about `pieces` pieces; built on first use and kept.
  const SlicedOp& sliced(uint32_t lw, uint32_t pieces, cudaStream_t s);
  OpView<double> rview64() const { return {n, nnz, relabel->off.get(), relabel->cols.get(), has_vals ? relabel->vals64.get() : nullptr}; }
  OpView<float> rview32() const { return {n, nnz, relabel->off.get(), relabel->cols.get(), has_vals ? relabel->vals32.get() : nullptr}; }
  OpView<double> view64() const { return {n, nnz, rows->off.get(), rows->tgt.get(), has_vals ? vals64.get() : nullptr}; }
  OpView<float> view32() const { return {n, nnz, rows->off.get(), rows->tgt.get(), has_vals ? vals32.get() : nullptr}; }
  const Partition& partition(uint32_t tile_items, cudaStream_t s);
};

struct GraphHandleImpl {
  uint32_t n = 0;
  uint64_t m = 0;
  bool directed = false;
  bool weighted = false;
  int device = 0;
  DevBuf<uint32_t> src, tgt;  // edges in input order
  DevBuf<double> w;
  std::vector<uint32_t> h_src, h_tgt;  // host copies (components, acyclicity)
  std::vector<double> h_w;
  DevCsr out;                  // out-arcs (all arcs for undirected graphs)
  DevCsr inc;                  // in-arcs, directed graphs only
  std::unique_ptr<DevCsr> und; // directions ignored, directed graphs only (lazy)
  std::mutex mu;               // guards the lazy members below and `und`
  // operators keyed by (which rows: 0 out, 1 in, 2 undirected; weighted; loop factor x 2)
  std::map<std::tuple<int, int, int>, std::unique_ptr<Operator>> ops;

  const DevCsr& in_rows() const { return directed ? inc : out; }
  const DevCsr& undirected_rows(cudaStream_t s);
  Operator& op(int which, bool weighted, double loop_factor, cudaStream_t s);
  // Operators whose arc values come from per-edge weights d_w (device,
  // input edge order) given per call, one per (rows, loop factor): the
  // structure, partitions and workspaces stay, and each call rewrites the
  // values (fill_weights) while it holds the slot's mutex.
  struct WeightSlot {
    std::mutex mu;
    std::unique_ptr<Operator> op;
  };
  std::map<std::pair<int, int>, std::unique_ptr<WeightSlot>> wslots;  // guarded by mu
  WeightSlot& weight_slot(int which, double loop_factor, cudaStream_t s);
  // Arc values, column sums and their inverses of o from d_w.
  void fill_weights(Operator& o, const double* d_w, double loop_factor, cudaStream_t s);
};

// Merge-path tile coordinates and split rows of a row-compressed matrix.
std::unique_ptr<Partition> build_partition(uint32_t n, uint64_t nnz, const uint32_t* off,
                                           uint32_t tile_items, cudaStream_t s);

// Builds the CSR of arcs (from[k], to[k]) whose payload edge[k] is the input
// edge; arcs must be listed in input order. Stable: ties keep that order.
void build_csr(uint32_t n, uint64_t arcs, const uint32_t* from, const uint32_t* to,
               const uint32_t* edge, const double* edge_w, DevCsr* out, cudaStream_t s);

// Undirected arcs of edges (src, tgt): each non-loop edge gives (s, t) then
// (t, s), a loop one arc (crates/engine/src/graph.rs:202-222).
void build_undirected(uint32_t n, uint64_t m, const uint32_t* src, const uint32_t* tgt,
                      const double* w, DevCsr* out, cudaStream_t s);

// Stable LSD radix sort of (keys, vals) by the low `bits` bits of the keys.
void radix_sort(uint64_t* keys, uint32_t* vals, size_t n, int bits, cudaStream_t s);

// Device-wide exclusive scan of n values (in may equal out); returns the total.
template <class T>
T exclusive_scan(const T* in, T* out, size_t n, cudaStream_t s);

cudaStream_t thread_stream();

}  // namespace knb
