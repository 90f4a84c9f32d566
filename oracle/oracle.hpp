// CPU oracle for the spectral-centrality path: TEST INFRASTRUCTURE ONLY.
//
// This is a plain C++ restatement of what knappnet's Rust engine computes on
// this path (graph build, degree, components, PageRank, eigenvector
// centrality by power iteration and thick-restart Lanczos, the EISPACK
// symmetric eigensolver, Philox random streams and the G(n, m) generator).
// Each function cites the reference file:line it follows. The reference
// itself cannot be compiled here (it is Rust and no Rust toolchain is
// present), so the oracle is pinned instead by the reference's golden files
// and known-answer tests (tests/test_oracle_golden.py).
//
// Only tests, the smoke check and the benchmark's CPU-baseline leg use this
// code, and only as the checker or the timed CPU baseline. The product
// library (knappnet_b200/) never links it.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace orc {

// ---------------------------------------------------------------- errors
struct Error {
  std::string msg;
};

// ---------------------------------------------------------------- random
// Philox4x32-10, crates/engine/src/rng.rs:10-34.
void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

// Stream(seed, index), crates/engine/src/rng.rs:36-97.
class Stream {
 public:
  Stream(uint64_t seed, uint64_t index);
  uint32_t next_u32();
  uint64_t next_u64();
  uint64_t below(uint64_t n);
  double uniform();

 private:
  uint32_t key_[2];
  uint64_t stream_;
  uint64_t block_ = 0;
  uint32_t buf_[4] = {0, 0, 0, 0};
  int used_ = 4;
};

// ---------------------------------------------------------------- graph
// One direction of adjacency, crates/engine/src/graph.rs:19-24.
struct Csr {
  std::vector<uint64_t> off;  // n + 1
  std::vector<uint32_t> tgt;  // arcs
  std::vector<double> w;      // arcs, empty when unweighted
  bool weighted = false;
  size_t n() const { return off.size() - 1; }
  size_t arcs() const { return tgt.size(); }
};

// graph.rs:121-133.
struct Graph {
  size_t n = 0;
  bool directed = false;
  std::vector<uint32_t> src, tgt;
  std::vector<double> w;
  bool weighted = false;
  Csr out;
  Csr inc;  // only for directed graphs
  const Csr& in_rows() const { return directed ? inc : out; }
};

Csr csr_build(size_t n, const uint32_t* from, const uint32_t* to, const double* w, size_t m);
Graph graph_from_edges(size_t n, const int64_t* src, const int64_t* tgt, const double* w,
                       size_t m, bool directed);

enum class Mode { Out = 1, In = 2, All = 3 };
Mode mode_from_code(int32_t code);

std::vector<double> degree(const Graph& g, Mode mode, bool loops, bool weighted);

// ---------------------------------------------------------------- components
struct Components {
  std::vector<uint32_t> membership;
  std::vector<size_t> sizes;
  size_t count() const { return sizes.size(); }
};
Components components(const Graph& g, bool strong);

// ---------------------------------------------------------------- operators
enum class Loops { Twice = 0, Once = 1, Ignore = 2 };
Loops loops_from_code(int32_t code);
double loop_factor(Loops l, bool directed);

// SparseOp, crates/engine/src/metrics/eigenvector.rs:498-704.
struct SparseOp {
  std::vector<uint64_t> off;
  std::vector<uint32_t> cols;
  std::vector<double> vals;  // empty when every entry is 1
  bool has_vals = false;
  size_t threads = 1;
  size_t dim() const { return off.size() - 1; }
  void apply(const double* x, double* y) const;
  void row_sums(size_t v, double* s, double* q) const;
  SparseOp submatrix(const std::vector<uint32_t>& rows, const std::vector<uint32_t>& col_index) const;
};
SparseOp op_from_rows(const Csr& rows, size_t dim, bool weighted, double loop_factor, size_t threads);

size_t threads_for(size_t requested, size_t items, uint64_t work);

// ---------------------------------------------------------------- measures
struct PagerankOptions {
  double damping = 0.85;
  bool directed = true;
  bool weighted = false;
  const double* personalization = nullptr;  // n values or null
  int dangling = 0;                          // 0 personalized, 1 uniform
  Loops loops = Loops::Twice;
  double tol = 1e-12;
  size_t max_iter = 10000;
  size_t threads = 0;
  size_t fixed_iters = 0;  // > 0: run exactly this many iterations (CPU timing only)
};
std::vector<double> pagerank(const Graph& g, const PagerankOptions& o, size_t* iters);

// The iteration of pagerank() on an operator already in pull form (rows = the
// arcs arriving at a node). Used by the CPU baseline on a prebuilt operator.
std::vector<double> pagerank_on_op(const SparseOp& op, const std::vector<double>& out_strength,
                                   double damping, const std::vector<double>& p,
                                   const std::vector<double>& jump, double tol, size_t max_iter,
                                   size_t fixed_iters, size_t* iters);

struct EigenvectorOptions {
  Mode mode = Mode::In;
  bool weighted = false;
  int scale = 0;  // 0 max, 1 unit
  Loops loops = Loops::Twice;
  double tol = 1e-12;
  size_t max_iter = 10000;
  size_t threads = 0;
};
struct Eigenvector {
  std::vector<double> values;
  double eigenvalue = 0;
  size_t iterations = 0;
  bool connected = true;
};
Eigenvector eigenvector_centrality(const Graph& g, const EigenvectorOptions& o);

// spectral.rs:308-344 (KatzOptions) and 555-594 (BonacichOptions).
struct KatzOptions {
  double alpha = 0.1;
  std::vector<double> beta{1.0};  // one value, or one per node
  Mode mode = Mode::In;
  bool weighted = false;
  Loops loops = Loops::Once;
  bool normalized = true;
  double tol = 1e-12;
  size_t max_iter = 10000;
  size_t threads = 0;
};
std::vector<double> katz(const Graph& g, const KatzOptions& o, size_t* iters);

struct BonacichOptions {
  double exponent = 1.0;
  Mode mode = Mode::Out;
  bool weighted = false;
  Loops loops = Loops::Ignore;
  bool rescale = false;
  double tol = 1e-12;
  size_t max_iter = 10000;
  size_t threads = 0;
};
std::vector<double> bonacich_power(const Graph& g, const BonacichOptions& o, size_t* iters,
                                   bool* dense);

// spectral.rs:676-746 (HitsScale, HitsOptions, Hits).
struct HitsOptions {
  bool weighted = false;
  Loops loops = Loops::Twice;
  int scale = 0;  // 0 largest 1, 1 sum 1, 2 unit norm
  double tol = 1e-12;
  size_t max_iter = 10000;
  size_t threads = 0;
};
struct Hits {
  std::vector<double> hubs, authorities;
  double value = 0;
  bool unique = false;
};
Hits hits(const Graph& g, const HitsOptions& o);

// linalg.rs:433-467: Gaussian elimination with partial pivoting on the
// row-major n x n matrix `a`; false when a pivot is at most tol times the
// largest magnitude of `a`.
bool dense_solve_rowmajor(std::vector<double> a, size_t n, std::vector<double>* x, double tol);

// linalg.rs:478-720: eigenvalues ascending, eigenvectors in columns of the
// row-major n x n matrix `vecs` (vecs[i * n + j] = component i of vector j).
bool symmetric_eigen(const std::vector<double>& a, size_t n, std::vector<double>* vals,
                     std::vector<double>* vecs);

// ---------------------------------------------------------------- generators
// G(n, m), crates/engine/src/generate.rs:255-290 with stream (seed, rep).
void gnm(size_t n, uint64_t m, bool directed, bool loops, uint64_t seed, uint64_t rep,
         std::vector<uint32_t>* from, std::vector<uint32_t>* to);

}  // namespace orc
