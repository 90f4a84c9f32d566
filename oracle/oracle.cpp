// CPU oracle for the spectral-centrality path: TEST INFRASTRUCTURE ONLY.
// See oracle.hpp for what this file is and is not. Every function restates
// the behaviour of the reference file:line it names, in code of its own.
#include "oracle.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <numeric>
#include <thread>
#include <unordered_set>

namespace orc {

static std::string fmt_g(double v) {
  char b[64];
  snprintf(b, sizeof b, "%g", v);
  return b;
}

// ======================================================== Philox and streams
// Salmon et al. 2011; the round function and constants are the published
// Philox4x32-10 (reference: crates/engine/src/rng.rs:10-34).
void philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    if (r) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

// rng.rs:46-56: key = seed halves, counter = (block, stream index).
Stream::Stream(uint64_t seed, uint64_t index) : stream_(index) {
  key_[0] = (uint32_t)seed;
  key_[1] = (uint32_t)(seed >> 32);
}

// rng.rs:58-74: four words per block, consumed in order.
uint32_t Stream::next_u32() {
  if (used_ == 4) {
    uint32_t ctr[4] = {(uint32_t)block_, (uint32_t)(block_ >> 32), (uint32_t)stream_,
                       (uint32_t)(stream_ >> 32)};
    philox4x32_10(ctr, key_, buf_);
    ++block_;
    used_ = 0;
  }
  return buf_[used_++];
}

// rng.rs:76-79: high word first.
uint64_t Stream::next_u64() {
  uint64_t hi = next_u32();
  uint64_t lo = next_u32();
  return hi << 32 | lo;
}

// rng.rs:81-92: rejection above the largest multiple of n.
uint64_t Stream::below(uint64_t n) {
  const uint64_t mx = std::numeric_limits<uint64_t>::max();
  uint64_t zone = mx - (mx % n + 1) % n;
  for (;;) {
    uint64_t x = next_u64();
    if (x <= zone) return x % n;
  }
}

// rng.rs:94-97: 53 random bits.
double Stream::uniform() { return (double)(next_u64() >> 11) * (1.0 / 9007199254740992.0); }

// ======================================================== graph build
// Stable two-pass counting sort, graph.rs:74-118: arcs ordered by source,
// then target, then input position.
Csr csr_build(size_t n, const uint32_t* from, const uint32_t* to, const double* w, size_t m) {
  std::vector<uint64_t> by_t(n + 1, 0);
  for (size_t a = 0; a < m; ++a) by_t[to[a] + 1]++;
  for (size_t i = 0; i < n; ++i) by_t[i + 1] += by_t[i];
  std::vector<uint64_t> order(m);
  {
    std::vector<uint64_t> cur(by_t.begin(), by_t.end() - 1);
    for (size_t a = 0; a < m; ++a) order[cur[to[a]]++] = a;
  }
  Csr c;
  c.off.assign(n + 1, 0);
  for (size_t a = 0; a < m; ++a) c.off[from[a] + 1]++;
  for (size_t i = 0; i < n; ++i) c.off[i + 1] += c.off[i];
  c.tgt.assign(m, 0);
  c.weighted = w != nullptr;
  if (w) c.w.assign(m, 0.0);
  std::vector<uint64_t> cur(c.off.begin(), c.off.end() - 1);
  for (size_t k = 0; k < m; ++k) {
    uint64_t a = order[k];
    uint64_t slot = cur[from[a]]++;
    c.tgt[slot] = to[a];
    if (w) c.w[slot] = w[a];
  }
  return c;
}

// graph.rs:142-234 (validation order and messages follow the reference's
// error kinds: node count, weights finite, edge count, endpoints).
Graph graph_from_edges(size_t n, const int64_t* src, const int64_t* tgt, const double* w,
                       size_t m, bool directed) {
  if (n > 0xFFFFFFFFull)
    throw Error{"node count (" + std::to_string(n) + ") exceeds the supported maximum"};
  if (w) {
    for (size_t e = 0; e < m; ++e)
      if (!std::isfinite(w[e]))
        throw Error{"edge " + std::to_string(e) + " has a missing, NaN, or infinite weight"};
  }
  if (m > 0xFFFFFFFFull / 2)
    throw Error{"edge count (" + std::to_string(m) + ") exceeds the supported maximum"};
  Graph g;
  g.n = n;
  g.directed = directed;
  g.src.resize(m);
  g.tgt.resize(m);
  for (size_t e = 0; e < m; ++e) {
    int64_t a = src[e], b = tgt[e];
    if (a < 0 || (uint64_t)a >= n)
      throw Error{"edge " + std::to_string(e) + " refers to node index " + std::to_string(a) +
                  ", but valid indices are 0.." + std::to_string(n)};
    g.src[e] = (uint32_t)a;
    if (b < 0 || (uint64_t)b >= n)
      throw Error{"edge " + std::to_string(e) + " refers to node index " + std::to_string(b) +
                  ", but valid indices are 0.." + std::to_string(n)};
    g.tgt[e] = (uint32_t)b;
  }
  g.weighted = w != nullptr;
  if (w) g.w.assign(w, w + m);
  if (directed) {
    g.out = csr_build(n, g.src.data(), g.tgt.data(), w ? g.w.data() : nullptr, m);
    g.inc = csr_build(n, g.tgt.data(), g.src.data(), w ? g.w.data() : nullptr, m);
  } else {
    // A non-loop edge becomes two arcs in a row, a loop one (graph.rs:202-222).
    std::vector<uint32_t> f, t;
    std::vector<double> ww;
    f.reserve(2 * m);
    t.reserve(2 * m);
    if (w) ww.reserve(2 * m);
    for (size_t e = 0; e < m; ++e) {
      f.push_back(g.src[e]);
      t.push_back(g.tgt[e]);
      if (w) ww.push_back(w[e]);
      if (g.src[e] != g.tgt[e]) {
        f.push_back(g.tgt[e]);
        t.push_back(g.src[e]);
        if (w) ww.push_back(w[e]);
      }
    }
    g.out = csr_build(n, f.data(), t.data(), w ? ww.data() : nullptr, f.size());
  }
  return g;
}

Mode mode_from_code(int32_t code) {
  if (code < 1 || code > 3) throw Error{"unknown degree mode code " + std::to_string(code)};
  return (Mode)code;
}

// metrics/degree.rs:41-73: per-edge endpoint counts in edge order.
std::vector<double> degree(const Graph& g, Mode mode, bool loops, bool weighted) {
  if (weighted && !g.weighted) throw Error{"the graph has no edge weights"};
  std::vector<double> out(g.n, 0.0);
  for (size_t e = 0; e < g.src.size(); ++e) {
    uint32_t s = g.src[e], t = g.tgt[e];
    if (s == t && !loops) continue;
    double x = weighted ? g.w[e] : 1.0;
    if (!g.directed) {
      out[s] += x;
      out[t] += x;
      continue;
    }
    if (mode != Mode::In) out[s] += x;
    if (mode != Mode::Out) out[t] += x;
  }
  return out;
}

// ======================================================== components
// Union-find with the smaller root kept and path halving (union_find.rs);
// weak components over the edge list (topography.rs:239-246).
static std::vector<uint32_t> weak_roots(const Graph& g) {
  std::vector<uint32_t> parent(g.n);
  std::iota(parent.begin(), parent.end(), 0u);
  auto find = [&](uint32_t v) {
    while (parent[v] != v) {
      parent[v] = parent[parent[v]];
      v = parent[v];
    }
    return v;
  };
  for (size_t e = 0; e < g.src.size(); ++e) {
    uint32_t a = find(g.src[e]), b = find(g.tgt[e]);
    if (a == b) continue;
    if (a < b) parent[b] = a; else parent[a] = b;
  }
  std::vector<uint32_t> r(g.n);
  for (uint32_t v = 0; v < g.n; ++v) r[v] = find(v);
  return r;
}

// Iterative Tarjan over out-arcs (topography.rs:248-305).
static std::vector<uint32_t> tarjan(const Graph& g) {
  const uint32_t UNSEEN = 0xFFFFFFFFu;
  size_t n = g.n;
  const Csr& adj = g.out;
  std::vector<uint32_t> index(n, UNSEEN), low(n, 0), comp(n, UNSEEN), stack;
  std::vector<uint8_t> on(n, 0);
  std::vector<std::pair<uint32_t, uint64_t>> frames;
  uint32_t counter = 0, ncomp = 0;
  for (size_t root = 0; root < n; ++root) {
    if (index[root] != UNSEEN) continue;
    frames.push_back({(uint32_t)root, 0});
    index[root] = low[root] = counter++;
    stack.push_back((uint32_t)root);
    on[root] = 1;
    while (!frames.empty()) {
      uint32_t v = frames.back().first;
      uint64_t& pos = frames.back().second;
      uint64_t deg = adj.off[v + 1] - adj.off[v];
      if (pos < deg) {
        uint32_t w = adj.tgt[adj.off[v] + pos];
        ++pos;
        if (index[w] == UNSEEN) {
          index[w] = low[w] = counter++;
          stack.push_back(w);
          on[w] = 1;
          frames.push_back({w, 0});
        } else if (on[w]) {
          low[v] = std::min(low[v], index[w]);
        }
        continue;
      }
      frames.pop_back();
      if (!frames.empty()) {
        uint32_t p = frames.back().first;
        low[p] = std::min(low[p], low[v]);
      }
      if (low[v] == index[v]) {
        for (;;) {
          uint32_t w = stack.back();
          stack.pop_back();
          on[w] = 0;
          comp[w] = ncomp;
          if (w == v) break;
        }
        ++ncomp;
      }
    }
  }
  return comp;
}

// topography.rs:183-207: relabel in order of first appearance.
Components components(const Graph& g, bool strong) {
  std::vector<uint32_t> raw = (strong && g.directed) ? tarjan(g) : weak_roots(g);
  Components c;
  std::vector<uint32_t> relabel(g.n, 0xFFFFFFFFu);
  c.membership.resize(g.n);
  for (size_t v = 0; v < g.n; ++v) {
    uint32_t r = raw[v];
    if (relabel[r] == 0xFFFFFFFFu) {
      relabel[r] = (uint32_t)c.sizes.size();
      c.sizes.push_back(0);
    }
    c.membership[v] = relabel[r];
    c.sizes[relabel[r]]++;
  }
  return c;
}

// ======================================================== operators
Loops loops_from_code(int32_t code) {
  if (code < 0 || code > 2) throw Error{"unknown self-loop weight code " + std::to_string(code)};
  return (Loops)code;
}

// eigenvector.rs:163-169.
double loop_factor(Loops l, bool directed) {
  if (l == Loops::Ignore) return 0.0;
  if (!directed && l == Loops::Twice) return 2.0;
  return 1.0;
}

// parallel.rs:29-55: all cores for 0, at most one thread per 2^17 steps.
size_t threads_for(size_t requested, size_t items, uint64_t work) {
  size_t avail = std::max(1u, std::thread::hardware_concurrency());
  size_t t = requested == 0 ? avail : requested;
  t = std::max<size_t>(1, std::min(t, std::max<size_t>(items, 1)));
  size_t by_work = (size_t)std::max<uint64_t>(1, work >> 17);
  return std::min(t, by_work);
}

// eigenvector.rs:512-547.
SparseOp op_from_rows(const Csr& rows, size_t dim, bool weighted, double lf, size_t threads) {
  SparseOp op;
  op.off.reserve(dim + 1);
  op.off.push_back(0);
  op.cols.reserve(rows.arcs());
  bool use_w = weighted && rows.weighted;
  op.has_vals = !(!use_w && lf == 1.0);
  if (op.has_vals) op.vals.reserve(rows.arcs());
  for (size_t v = 0; v < dim; ++v) {
    for (uint64_t k = rows.off[v]; k < rows.off[v + 1]; ++k) {
      uint32_t j = rows.tgt[k];
      op.cols.push_back(j);
      if (op.has_vals) {
        double x = use_w ? rows.w[k] : 1.0;
        op.vals.push_back(j == v ? x * lf : x);
      }
    }
    op.off.push_back(op.cols.size());
  }
  op.threads = threads_for(threads, dim, op.cols.size() / 2);
  return op;
}

// eigenvector.rs:659-703: one sum per row in CSR order; threads take
// contiguous blocks of rows, so the result does not depend on their count.
void SparseOp::apply(const double* x, double* y) const {
  size_t n = dim();
  auto rows = [&](size_t lo, size_t hi) {
    for (size_t v = lo; v < hi; ++v) {
      double acc = 0.0;
      if (!has_vals) {
        for (uint64_t k = off[v]; k < off[v + 1]; ++k) acc += x[cols[k]];
      } else {
        for (uint64_t k = off[v]; k < off[v + 1]; ++k) acc += vals[k] * x[cols[k]];
      }
      y[v] = acc;
    }
  };
  if (threads <= 1) {
    rows(0, n);
    return;
  }
  size_t block = (n + threads - 1) / threads;
  std::vector<std::thread> pool;
  for (size_t b = 0; b < threads; ++b) {
    size_t lo = std::min(b * block, n), hi = std::min((b + 1) * block, n);
    pool.emplace_back(rows, lo, hi);
  }
  for (auto& t : pool) t.join();
}

// eigenvector.rs:566-584: row sum, and sum of squares with parallel entries
// (adjacent in a sorted row) merged first.
void SparseOp::row_sums(size_t v, double* s_out, double* q_out) const {
  double s = 0, q = 0;
  bool have = false;
  uint32_t c = 0;
  double acc = 0;
  for (uint64_t k = off[v]; k < off[v + 1]; ++k) {
    uint32_t j = cols[k];
    double w = has_vals ? vals[k] : 1.0;
    s += w;
    if (have && c == j) {
      acc += w;
    } else {
      if (have) q += acc * acc;
      c = j;
      acc = w;
      have = true;
    }
  }
  if (have) q += acc * acc;
  *s_out = s;
  *q_out = q;
}

// eigenvector.rs:598-624.
SparseOp SparseOp::submatrix(const std::vector<uint32_t>& rows,
                             const std::vector<uint32_t>& col_index) const {
  SparseOp s;
  s.has_vals = has_vals;
  s.off.push_back(0);
  for (uint32_t v : rows) {
    for (uint64_t k = off[v]; k < off[v + 1]; ++k) {
      uint32_t c = col_index[cols[k]];
      if (c == 0xFFFFFFFFu) continue;
      s.cols.push_back(c);
      if (has_vals) s.vals.push_back(vals[k]);
    }
    s.off.push_back(s.cols.size());
  }
  s.threads = threads_for(std::max<size_t>(threads, 1), rows.size(), s.cols.size() / 2);
  return s;
}

// ======================================================== PageRank
// spectral.rs:163-170.
static void check_iteration(double tol, size_t max_iter) {
  if (std::isnan(tol) || tol <= 0.0 || max_iter == 0)
    throw Error{"the tolerance and the iteration cap must be positive"};
}

// weights.rs:137-149 via eigenvector.rs:323-325.
static void check_nonnegative(const Graph& g, const char* what) {
  if (!g.weighted) throw Error{"the graph has no edge weights"};
  for (size_t e = 0; e < g.w.size(); ++e)
    if (g.w[e] < 0.0)
      throw Error{"edge " + std::to_string(e) + " has negative weight " + fmt_g(g.w[e]) + "; " +
                  what + " requires non-negative weights"};
}

// spectral.rs:284-304.
static std::vector<double> probabilities(const double* p, size_t n, const char* what) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i]) || p[i] < 0.0)
      throw Error{std::string("the ") + what + " vector must hold finite, nonnegative values"};
  double total = 0;
  for (size_t i = 0; i < n; ++i) total += p[i];
  if (total <= 0.0) throw Error{std::string("the ") + what + " vector must have a positive sum"};
  std::vector<double> r(n);
  for (size_t i = 0; i < n; ++i) r[i] = p[i] / total;
  return r;
}

// closeness.rs:224-236 + spectral.rs:174-208: the rows a measure follows.
// Returns the undirected rebuild through `holder` when one is needed.
static const Graph& oriented(const Graph& g, Mode mode, Graph* holder) {
  if (!g.directed || mode == Mode::Out) return g;
  std::vector<int64_t> s(g.src.begin(), g.src.end()), t(g.tgt.begin(), g.tgt.end());
  const double* w = g.weighted ? g.w.data() : nullptr;
  if (mode == Mode::In)
    *holder = graph_from_edges(g.n, t.data(), s.data(), w, s.size(), true);
  else
    *holder = graph_from_edges(g.n, s.data(), t.data(), w, s.size(), false);
  return *holder;
}

static SparseOp matrix(const Graph& g, Mode mode, bool weighted, Loops loops, size_t threads,
                       Graph* holder) {
  if (!g.directed) mode = Mode::All;
  const Graph& h = oriented(g, mode == Mode::All ? Mode::All : Mode::Out, holder);
  const Csr& rows = (h.directed && mode == Mode::In) ? h.inc : h.out;
  return op_from_rows(rows, g.n, weighted, loop_factor(loops, h.directed), threads);
}

// spectral.rs:240-280 on a prepared operator.
std::vector<double> pagerank_on_op(const SparseOp& op, const std::vector<double>& out,
                                   double d, const std::vector<double>& p,
                                   const std::vector<double>& jump, double tol, size_t max_iter,
                                   size_t fixed_iters, size_t* iters) {
  size_t n = op.dim();
  std::vector<double> x(n, 1.0 / (double)n), z(n, 0.0), y(n, 0.0);
  size_t cap = fixed_iters ? fixed_iters : max_iter;
  for (size_t it = 0; it < cap; ++it) {
    double stuck = 0.0;
    for (size_t j = 0; j < n; ++j) {
      if (out[j] > 0.0) {
        z[j] = x[j] / out[j];
      } else {
        z[j] = 0.0;
        stuck += x[j];
      }
    }
    op.apply(z.data(), y.data());
    double total = 0.0;
    for (size_t i = 0; i < n; ++i) {
      y[i] = d * (y[i] + stuck * jump[i]) + (1.0 - d) * p[i];
      total += y[i];
    }
    double change = 0.0;
    for (size_t i = 0; i < n; ++i) {
      y[i] /= total;
      change += std::fabs(y[i] - x[i]);
    }
    std::swap(x, y);
    if (!fixed_iters && change <= tol) {
      if (iters) *iters = it + 1;
      return x;
    }
  }
  if (fixed_iters) {
    if (iters) *iters = fixed_iters;
    return x;
  }
  throw Error{"PageRank did not converge to tolerance " + fmt_g(tol) + " within " +
              std::to_string(max_iter) + " iterations"};
}

// spectral.rs:211-281.
std::vector<double> pagerank(const Graph& g, const PagerankOptions& o, size_t* iters) {
  check_iteration(o.tol, o.max_iter);
  if (!(o.damping >= 0.0 && o.damping <= 1.0))
    throw Error{"damping is " + fmt_g(o.damping) + "; it must be between 0 and 1"};
  size_t n = g.n;
  if (iters) *iters = 0;
  if (n == 0) return {};
  if (o.weighted) check_nonnegative(g, "PageRank");
  std::vector<double> p = o.personalization ? probabilities(o.personalization, n, "personalization")
                                            : std::vector<double>(n, 1.0 / (double)n);
  std::vector<double> jump = o.dangling == 0 ? p : std::vector<double>(n, 1.0 / (double)n);
  Graph holder;
  SparseOp op = matrix(g, o.directed ? Mode::In : Mode::All, o.weighted, o.loops, o.threads,
                       &holder);
  std::vector<double> out(n, 0.0);
  for (size_t i = 0; i < n; ++i)
    for (uint64_t k = op.off[i]; k < op.off[i + 1]; ++k)
      out[op.cols[k]] += op.has_vals ? op.vals[k] : 1.0;
  return pagerank_on_op(op, out, o.damping, p, jump, o.tol, o.max_iter, o.fixed_iters, iters);
}

// ======================================================== dense eigensolver
// Householder tridiagonalisation and implicit QL with accumulated
// transformations, in EISPACK's operation order (tred2/tql2; the reference
// follows the same order in linalg.rs:478-720). v is row-major n x n.
static void tred2(std::vector<double>& V, std::vector<double>& d, std::vector<double>& e, size_t n) {
  auto A = [&](size_t r, size_t c) -> double& { return V[r * n + c]; };
  for (size_t j = 0; j < n; ++j) d[j] = A(n - 1, j);
  for (size_t i = n - 1; i > 0; --i) {
    double scale = 0.0, h = 0.0;
    for (size_t k = 0; k < i; ++k) scale += std::fabs(d[k]);
    if (scale == 0.0) {
      e[i] = d[i - 1];
      for (size_t j = 0; j < i; ++j) {
        d[j] = A(i - 1, j);
        A(i, j) = 0.0;
        A(j, i) = 0.0;
      }
    } else {
      for (size_t k = 0; k < i; ++k) {
        d[k] /= scale;
        h += d[k] * d[k];
      }
      double f = d[i - 1];
      double g = std::sqrt(h);
      if (f > 0) g = -g;
      e[i] = scale * g;
      h -= f * g;
      d[i - 1] = f - g;
      for (size_t j = 0; j < i; ++j) e[j] = 0.0;
      for (size_t j = 0; j < i; ++j) {
        f = d[j];
        A(j, i) = f;
        g = e[j] + A(j, j) * f;
        for (size_t k = j + 1; k < i; ++k) {
          g += A(k, j) * d[k];
          e[k] += A(k, j) * f;
        }
        e[j] = g;
      }
      f = 0.0;
      for (size_t j = 0; j < i; ++j) {
        e[j] /= h;
        f += e[j] * d[j];
      }
      double hh = f / (h + h);
      for (size_t j = 0; j < i; ++j) e[j] -= hh * d[j];
      for (size_t j = 0; j < i; ++j) {
        f = d[j];
        g = e[j];
        for (size_t k = j; k < i; ++k) A(k, j) -= (f * e[k] + g * d[k]);
        d[j] = A(i - 1, j);
        A(i, j) = 0.0;
      }
    }
    d[i] = h;
  }
  for (size_t i = 0; i + 1 < n; ++i) {
    A(n - 1, i) = A(i, i);
    A(i, i) = 1.0;
    double h = d[i + 1];
    if (h != 0.0) {
      for (size_t k = 0; k <= i; ++k) d[k] = A(k, i + 1) / h;
      for (size_t j = 0; j <= i; ++j) {
        double g = 0.0;
        for (size_t k = 0; k <= i; ++k) g += A(k, i + 1) * A(k, j);
        for (size_t k = 0; k <= i; ++k) A(k, j) -= g * d[k];
      }
    }
    for (size_t k = 0; k <= i; ++k) A(k, i + 1) = 0.0;
  }
  for (size_t j = 0; j < n; ++j) {
    d[j] = A(n - 1, j);
    A(n - 1, j) = 0.0;
  }
  A(n - 1, n - 1) = 1.0;
  e[0] = 0.0;
}

static bool tql2(std::vector<double>& V, std::vector<double>& d, std::vector<double>& e, size_t n) {
  auto A = [&](size_t r, size_t c) -> double& { return V[r * n + c]; };
  for (size_t i = 1; i < n; ++i) e[i - 1] = e[i];
  e[n - 1] = 0.0;
  double f = 0.0, tst1 = 0.0;
  const double eps = std::numeric_limits<double>::epsilon();
  for (size_t l = 0; l < n; ++l) {
    tst1 = std::max(tst1, std::fabs(d[l]) + std::fabs(e[l]));
    size_t m = l;
    while (m < n) {
      if (std::fabs(e[m]) <= eps * tst1) break;
      ++m;
    }
    if (m > l) {
      int iter = 0;
      for (;;) {
        if (++iter > 60) return false;
        double g = d[l];
        double p = (d[l + 1] - g) / (2.0 * e[l]);
        double r = std::hypot(p, 1.0);
        if (p < 0) r = -r;
        d[l] = e[l] / (p + r);
        d[l + 1] = e[l] * (p + r);
        double dl1 = d[l + 1];
        double h = g - d[l];
        for (size_t i = l + 2; i < n; ++i) d[i] -= h;
        f += h;
        p = d[m];
        double c = 1.0, c2 = c, c3 = c;
        double el1 = e[l + 1];
        double s = 0.0, s2 = 0.0;
        for (size_t i = m; i-- > l;) {
          c3 = c2;
          c2 = c;
          s2 = s;
          g = c * e[i];
          h = c * p;
          r = std::hypot(p, e[i]);
          e[i + 1] = s * r;
          s = e[i] / r;
          c = p / r;
          p = c * d[i] - s * g;
          d[i + 1] = h + s * (c * g + s * d[i]);
          for (size_t k = 0; k < n; ++k) {
            h = A(k, i + 1);
            A(k, i + 1) = s * A(k, i) + c * h;
            A(k, i) = c * A(k, i) - s * h;
          }
        }
        p = -s * s2 * c3 * el1 * e[l] / dl1;
        e[l] = s * p;
        d[l] = c * p;
        if (std::fabs(e[l]) <= eps * tst1) break;
      }
    }
    d[l] += f;
    e[l] = 0.0;
  }
  for (size_t i = 0; i + 1 < n; ++i) {
    size_t k = i;
    double p = d[i];
    for (size_t j = i + 1; j < n; ++j)
      if (d[j] < p) {
        k = j;
        p = d[j];
      }
    if (k != i) {
      d[k] = d[i];
      d[i] = p;
      for (size_t r = 0; r < n; ++r) std::swap(A(r, i), A(r, k));
    }
  }
  return true;
}

bool symmetric_eigen(const std::vector<double>& a, size_t n, std::vector<double>* vals,
                     std::vector<double>* vecs) {
  vals->assign(n, 0.0);
  *vecs = a;
  if (n == 0) return true;
  std::vector<double> e(n, 0.0);
  tred2(*vecs, *vals, e, n);
  return tql2(*vecs, *vals, e, n);
}

// ======================================================== Lanczos
// Constants of eigenvector.rs:729-740.
static const size_t MAX_BASIS = 20;
static const size_t KEEP = 8;
static const size_t MAX_BASIS_DOUBLES = (size_t)1 << 27;
static const size_t BLOCK = 4096;
static const size_t CHECK_EVERY = 4;

// Sums over fixed 4096-row blocks added in block order (eigenvector.rs:913-971).
struct Blocks {
  size_t dim, count;
  explicit Blocks(size_t d) : dim(d), count((d + BLOCK - 1) / BLOCK) {}
  double dot(const double* a, const double* b) const {
    double total = 0.0;
    for (size_t bk = 0; bk < count; ++bk) {
      double s = 0.0;
      for (size_t i = bk * BLOCK, e = std::min(dim, (bk + 1) * BLOCK); i < e; ++i) s += a[i] * b[i];
      total += s;
    }
    return total;
  }
  double sum(const double* a) const {
    double total = 0.0;
    for (size_t bk = 0; bk < count; ++bk) {
      double s = 0.0;
      for (size_t i = bk * BLOCK, e = std::min(dim, (bk + 1) * BLOCK); i < e; ++i) s += a[i];
      total += s;
    }
    return total;
  }
};

// Basis vectors stored one after another (eigenvector.rs:975-1122).
struct Basis {
  size_t dim;
  std::vector<double> data;
  const double* col(size_t l) const { return data.data() + l * dim; }
  double* col(size_t l) { return data.data() + l * dim; }
  void set_col(size_t l, const std::vector<double>& v) { std::copy(v.begin(), v.end(), col(l)); }

  std::vector<double> project(size_t lo, size_t hi, const double* w, const Blocks& b) const {
    std::vector<double> total(hi - lo, 0.0);
    for (size_t bk = 0; bk < b.count; ++bk) {
      size_t r0 = bk * BLOCK, r1 = std::min(dim, (bk + 1) * BLOCK);
      for (size_t l = lo; l < hi; ++l) {
        const double* v = col(l);
        double s = 0.0;
        for (size_t i = r0; i < r1; ++i) s += v[i] * w[i];
        total[l - lo] += s;
      }
    }
    return total;
  }
  double subtract(size_t lo, size_t hi, const std::vector<double>& h, double* w,
                  const Blocks& b) const {
    double total = 0.0;
    for (size_t bk = 0; bk < b.count; ++bk) {
      size_t r0 = bk * BLOCK, r1 = std::min(dim, (bk + 1) * BLOCK);
      for (size_t l = lo; l < hi; ++l) {
        const double* v = col(l);
        double c = h[l - lo];
        for (size_t i = r0; i < r1; ++i) w[i] -= c * v[i];
      }
      double sq = 0.0;
      for (size_t i = r0; i < r1; ++i) sq += w[i] * w[i];
      total += sq;
    }
    return std::sqrt(total);
  }
  // Classical Gram-Schmidt against the last two vectors, then full passes
  // under the DGKS test (eigenvector.rs:997-1021).
  void orthogonalize(size_t cols, double* w, const Blocks& b, std::vector<double>* coef,
                     double* before_out, double* after_out) const {
    double before = std::sqrt(b.dot(w, w));
    size_t lo = cols >= 2 ? cols - 2 : 0;
    coef->assign(cols, 0.0);
    std::vector<double> local = project(lo, cols, w, b);
    double mid = subtract(lo, cols, local, w, b);
    for (size_t l = lo; l < cols; ++l) (*coef)[l] += local[l - lo];
    for (;;) {
      std::vector<double> again = project(0, cols, w, b);
      double after = subtract(0, cols, again, w, b);
      for (size_t l = 0; l < cols; ++l) (*coef)[l] += again[l];
      if (after >= M_SQRT1_2 * mid || after == 0.0 || mid == before) {
        *before_out = before;
        *after_out = after;
        return;
      }
      mid = before;
    }
  }
  std::vector<double> combine(size_t cols, const std::vector<double>& s) const {
    std::vector<double> out(dim, 0.0);
    for (size_t l = 0; l < cols; ++l) {
      const double* v = col(l);
      double c = s[l];
      for (size_t i = 0; i < dim; ++i) out[i] += c * v[i];
    }
    return out;
  }
  void rotate(size_t cols, const std::vector<double>& s, size_t p) {
    std::vector<double> out(p * dim, 0.0);
    for (size_t l = 0; l < cols; ++l) {
      const double* v = col(l);
      for (size_t q = 0; q < p; ++q) {
        double c = s[l * p + q];
        double* o = out.data() + q * dim;
        for (size_t i = 0; i < dim; ++i) o[i] += c * v[i];
      }
    }
    std::copy(out.begin(), out.end(), data.begin());
  }
};

struct Leading {
  double value;
  std::vector<double> vector;
  size_t matvecs;
};

static bool projected_eigen(const std::vector<double>& hm, size_t stride, size_t size,
                            std::vector<double>* theta, std::vector<double>* s) {
  std::vector<double> b(size * size);
  for (size_t i = 0; i < size; ++i)
    for (size_t j = 0; j < size; ++j) b[i * size + j] = 0.5 * (hm[i * stride + j] + hm[j * stride + i]);
  return symmetric_eigen(b, size, theta, s);
}

static Leading finish_vector(std::vector<double> x, double value, size_t matvecs, const Blocks& b) {
  double total = b.sum(x.data());
  if (total < 0.0)
    for (double& v : x) v = -v;
  for (double& v : x)
    if (v < 0.0) v = 0.0;
  double norm = std::sqrt(b.dot(x.data(), x.data()));
  if (norm > 0.0)
    for (double& v : x) v /= norm;
  return Leading{value, std::move(x), matvecs};
}

// eigenvector.rs:746-878: the operator is given as `apply` (y = M x) on
// vectors of `dim` entries.
using Apply = std::function<void(const double*, double*)>;
static bool symmetric_leading(size_t dim, const Apply& apply, const std::vector<double>& start,
                              double tol, double shift, size_t max_matvecs, Leading* res) {
  size_t m = std::max<size_t>(
      1, std::min(std::min(dim, MAX_BASIS), std::max<size_t>(MAX_BASIS_DOUBLES / dim, 8)));
  size_t keep = std::max<size_t>(1, std::min(KEEP, m >= 2 ? m - 2 : 0));
  Blocks blocks(dim);
  Basis basis{dim, std::vector<double>(dim * m, 0.0)};
  std::vector<double> hm(m * m, 0.0);
  std::vector<double> v = start;
  double norm = std::sqrt(blocks.dot(v.data(), v.data()));
  if (norm == 0.0 || !std::isfinite(norm)) return false;
  for (double& x : v) x /= norm;
  basis.set_col(0, v);
  std::vector<double> w(dim, 0.0), y(dim, 0.0), coef, theta, s;
  size_t matvecs = 0, j0 = 0;
  double threshold = std::numeric_limits<double>::infinity();
  for (;;) {
    size_t j = j0;
    bool restart = false;
    while (!restart) {
      if (matvecs >= max_matvecs) return false;
      apply(v.data(), w.data());
      ++matvecs;
      double before, beta;
      basis.orthogonalize(j + 1, w.data(), blocks, &coef, &before, &beta);
      for (size_t i = 0; i < coef.size(); ++i) {
        hm[i * m + j] = coef[i];
        hm[j * m + i] = coef[i];
      }
      size_t size = j + 1;
      bool breakdown = beta <= 1e-12 * before || std::isnan(beta);
      bool end = breakdown || size == m;
      if (end || (size - j0) % CHECK_EVERY == 0) {
        if (!projected_eigen(hm, m, size, &theta, &s)) return false;
        size_t top = 0;
        for (size_t i = 0; i < size; ++i)
          if (theta[i] > theta[top]) top = i;
        double estimate = breakdown ? 0.0 : beta * std::fabs(s[(size - 1) * size + top]);
        double limit = tol * (std::max(theta[top], 0.0) + shift);
        if (estimate <= std::min(limit, threshold)) {
          std::vector<double> cf(size);
          for (size_t l = 0; l < size; ++l) cf[l] = s[l * size + top];
          std::vector<double> x = basis.combine(size, cf);
          if (matvecs >= max_matvecs) return false;
          apply(x.data(), y.data());
          ++matvecs;
          double xx = blocks.dot(x.data(), x.data());
          double value = blocks.dot(x.data(), y.data()) / xx;
          double rinf = 0.0, xinf = 0.0;
          for (size_t i = 0; i < dim; ++i) {
            rinf = std::max(rinf, std::fabs(y[i] - value * x[i]));
            xinf = std::max(xinf, std::fabs(x[i]));
          }
          double need = tol * (std::max(value, 0.0) + shift) * xinf;
          if (rinf <= need) {
            *res = finish_vector(std::move(x), value, matvecs, blocks);
            return true;
          }
          threshold = rinf > 0.0 ? std::min(estimate, limit) * (need / rinf) * 0.5
                                 : std::min(estimate, limit) * 0.5;
          if (breakdown) {
            double nx = std::sqrt(xx);
            for (size_t i = 0; i < dim; ++i) v[i] = x[i] / nx;
            basis.set_col(0, v);
            std::fill(hm.begin(), hm.end(), 0.0);
            j0 = 0;
            restart = true;
            continue;
          }
        }
        if (end) {
          if (breakdown) return false;
          std::vector<size_t> idx(size);
          std::iota(idx.begin(), idx.end(), 0);
          std::stable_sort(idx.begin(), idx.end(),
                           [&](size_t a_, size_t b_) { return theta[a_] > theta[b_]; });
          size_t p = std::min(keep, size - 1);
          std::vector<double> svec(size * p);
          for (size_t q = 0; q < p; ++q)
            for (size_t l = 0; l < size; ++l) svec[l * p + q] = s[l * size + idx[q]];
          basis.rotate(size, svec, p);
          std::fill(hm.begin(), hm.end(), 0.0);
          for (size_t q = 0; q < p; ++q) {
            hm[q * m + q] = theta[idx[q]];
            double c = beta * s[(size - 1) * size + idx[q]];
            hm[q * m + p] = c;
            hm[p * m + q] = c;
          }
          for (size_t i = 0; i < dim; ++i) v[i] = w[i] / beta;
          basis.set_col(p, v);
          j0 = p;
          restart = true;
          continue;
        }
      }
      for (size_t i = 0; i < dim; ++i) v[i] = w[i] / beta;
      basis.set_col(j + 1, v);
      hm[(j + 1) * m + j] = beta;
      hm[j * m + j + 1] = beta;
      ++j;
    }
  }
}

// eigenvector.rs:330-374.
static std::vector<double> power_iteration(const SparseOp& op, const EigenvectorOptions& o,
                                           double* lambda_out, size_t* iters) {
  size_t n = op.dim();
  std::vector<double> x(n, 1.0), y(n, 0.0);
  for (size_t it = 1; it <= o.max_iter; ++it) {
    op.apply(x.data(), y.data());
    double top = 0.0;
    for (size_t v = 0; v < n; ++v) {
      y[v] += x[v];
      top = std::max(top, y[v]);
    }
    double change = 0.0;
    for (size_t v = 0; v < n; ++v) {
      y[v] /= top;
      change = std::max(change, std::fabs(y[v] - x[v]));
    }
    std::swap(x, y);
    if (change <= o.tol) {
      op.apply(x.data(), y.data());
      double s0 = 0, s1 = 0, s2 = 0;
      for (size_t v = 0; v < n; ++v) {
        s0 += y[v];
        s1 += x[v];
        s2 += x[v] * x[v];
      }
      *lambda_out = s1 > 0.0 ? s0 / s1 : 0.0;
      if (s2 > 0.0) {
        double w = s1 / s2;
        for (double& xv : x) xv *= w;
      }
      *iters = it;
      return x;
    }
  }
  throw Error{"eigenvector centrality did not converge to tolerance " + fmt_g(o.tol) + " within " +
              std::to_string(o.max_iter) +
              " iterations. Power iteration converges slowly when the largest eigenvalue is "
              "close to the next one, and not at all to a single answer when several strongly "
              "connected components share it; a larger iteration cap may help in the first case"};
}

static const double TIE = 1e-9;

// eigenvector.rs:383-479.
static std::vector<double> symmetric_components(const Graph& h, const SparseOp& op,
                                                const EigenvectorOptions& o, double* best_out,
                                                size_t* matvecs_out) {
  size_t n = op.dim();
  Components comps = components(h, false);
  size_t k = comps.count();
  std::vector<double> upper(k, 0.0), sum(k, 0.0), square(k, 0.0);
  for (size_t v = 0; v < n; ++v) {
    uint32_t c = comps.membership[v];
    double s, q;
    op.row_sums(v, &s, &q);
    upper[c] = std::max(upper[c], s);
    sum[c] += s;
    square[c] = std::max(square[c], q);
  }
  std::vector<double> lower(k);
  for (size_t c = 0; c < k; ++c) lower[c] = std::max(sum[c] / (double)comps.sizes[c], std::sqrt(square[c]));
  std::vector<size_t> order(k);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t b) { return lower[b] < lower[a]; });
  std::vector<size_t> start(k + 1, 0);
  for (uint32_t c : comps.membership) start[c + 1]++;
  for (size_t c = 0; c < k; ++c) start[c + 1] += start[c];
  std::vector<uint32_t> members(n);
  {
    std::vector<size_t> cur(start.begin(), start.end() - 1);
    for (size_t v = 0; v < n; ++v) members[cur[comps.membership[v]]++] = (uint32_t)v;
  }
  double best = 0.0;
  size_t matvecs = 0;
  struct Solved {
    size_t c;
    double value;
    std::vector<double> u;
  };
  std::vector<Solved> solved;
  std::vector<uint32_t> local(n, 0);
  for (size_t c : order) {
    if (upper[c] <= 0.0 || upper[c] < best * (1.0 - TIE)) continue;
    std::vector<uint32_t> nodes(members.begin() + start[c], members.begin() + start[c + 1]);
    SparseOp sub;
    const SparseOp* a = &op;
    if (k != 1) {
      for (size_t i = 0; i < nodes.size(); ++i) local[nodes[i]] = (uint32_t)i;
      sub = op.submatrix(nodes, local);
      a = &sub;
    }
    std::vector<double> ones(nodes.size(), 1.0);
    Leading res;
    if (!symmetric_leading(a->dim(), [a](const double* x, double* y) { a->apply(x, y); }, ones,
                           o.tol, 1.0, o.max_iter, &res))
      throw Error{"eigenvector centrality did not converge to tolerance " + fmt_g(o.tol) +
                  " within " + std::to_string(o.max_iter) +
                  " matrix-vector products; a larger iteration cap may help"};
    matvecs += res.matvecs;
    best = std::max(best, res.value);
    solved.push_back({c, res.value, std::move(res.vector)});
  }
  std::vector<double> x(n, 0.0);
  for (auto& sv : solved) {
    if (sv.value < best * (1.0 - TIE)) continue;
    double total = 0.0;
    for (double u : sv.u) total += u;
    for (size_t i = start[sv.c]; i < start[sv.c + 1]; ++i) x[members[i]] = sv.u[i - start[sv.c]] * total;
  }
  *best_out = best;
  *matvecs_out = matvecs;
  return x;
}

// eigenvector.rs:481-491.
static void scale_vec(std::vector<double>& x, int how) {
  double d = 0.0;
  if (how == 0) {
    for (double v : x) d = std::max(d, v);
  } else {
    for (double v : x) d += v * v;
    d = std::sqrt(d);
  }
  if (d > 0.0)
    for (double& v : x) v /= d;
}

// eigenvector.rs:229-320.
Eigenvector eigenvector_centrality(const Graph& g, const EigenvectorOptions& o) {
  if (std::isnan(o.tol) || o.tol <= 0.0 || o.max_iter == 0)
    throw Error{"the tolerance and the iteration cap must be positive"};
  Eigenvector r;
  size_t n = g.n;
  if (n == 0) {
    r.eigenvalue = std::numeric_limits<double>::quiet_NaN();
    r.connected = true;
    return r;
  }
  if (o.weighted) check_nonnegative(g, "eigenvector centrality");
  Mode mode = g.directed ? o.mode : Mode::All;
  Graph holder;
  const Graph& h = oriented(g, mode == Mode::All ? Mode::All : Mode::Out, &holder);
  const Csr& rows = (h.directed && mode == Mode::In) ? h.inc : h.out;
  SparseOp op = op_from_rows(rows, n, o.weighted, loop_factor(o.loops, h.directed), o.threads);
  r.connected = components(h, h.directed).count() == 1;
  Components strong = components(h, true);
  bool cyclic = false;
  for (size_t v = 0; v < n && !cyclic; ++v)
    for (uint64_t k = op.off[v]; k < op.off[v + 1]; ++k) {
      double w = op.has_vals ? op.vals[k] : 1.0;
      if (strong.membership[op.cols[k]] == strong.membership[v] && w > 0.0) {
        cyclic = true;
        break;
      }
    }
  if (!cyclic) {
    std::vector<double> sink(n, 1.0);
    for (size_t v = 0; v < n; ++v)
      for (uint64_t k = op.off[v]; k < op.off[v + 1]; ++k)
        if ((op.has_vals ? op.vals[k] : 1.0) > 0.0) sink[op.cols[k]] = 0.0;
    scale_vec(sink, o.scale);
    r.values = std::move(sink);
    r.eigenvalue = 0.0;
    r.iterations = 0;
    return r;
  }
  if (h.directed) {
    r.values = power_iteration(op, o, &r.eigenvalue, &r.iterations);
  } else {
    r.values = symmetric_components(h, op, o, &r.eigenvalue, &r.iterations);
  }
  scale_vec(r.values, o.scale);
  return r;
}

// ======================================================== Katz, Bonacich
// spectral.rs:409-445: x = b + t A x by fixed-point iteration; stops when
// the change times q / (1 - q) (at least 1) is at most tol times the
// largest |x_i|, or when every score is 0.
static std::vector<double> solve_series(const SparseOp& op, const std::vector<double>& b, double t,
                                        double q, double tol, size_t max_iter, const char* what,
                                        size_t* iters) {
  const size_t n = b.size();
  std::vector<double> x = b;
  *iters = 0;
  if (t == 0.0) return x;
  const double factor = std::max(q / (1.0 - q), 1.0);
  std::vector<double> y(n, 0.0);
  for (size_t it = 0; it < max_iter; ++it) {
    op.apply(x.data(), y.data());
    double change = 0.0, top = 0.0;
    for (size_t i = 0; i < n; ++i) {
      y[i] = b[i] + t * y[i];
      change = std::max(change, std::fabs(y[i] - x[i]));
      top = std::max(top, std::fabs(y[i]));
    }
    std::swap(x, y);
    *iters = it + 1;
    if (change * factor <= tol * top || top == 0.0) return x;
  }
  throw Error{std::string(what) + " did not converge to tolerance " + fmt_g(tol) + " within " +
              std::to_string(max_iter) + " iterations"};
}

// spectral.rs:529-537.
static Error too_large(const char* name, double t, double lambda) {
  return Error{std::string(name) + " = " + fmt_g(t) +
               " is not below 1 / lambda_max: the largest eigenvalue of the adjacency matrix "
               "is at least " + fmt_g(lambda) + ", so 1 / lambda_max is at most " +
               fmt_g(1.0 / lambda)};
}

// spectral.rs:539-553: arcs i -> j for each positive entry (i, j).
static Graph pattern_graph(const SparseOp& op) {
  const size_t n = op.dim();
  std::vector<int64_t> s, t;
  for (size_t i = 0; i < n; ++i)
    for (uint64_t k = op.off[i]; k < op.off[i + 1]; ++k)
      if ((op.has_vals ? op.vals[k] : 1.0) > 0.0) {
        s.push_back((int64_t)i);
        t.push_back((int64_t)op.cols[k]);
      }
  return graph_from_edges(n, s.data(), t.data(), nullptr, s.size(), true);
}

// spectral.rs:447-527: checks that t times the spectral radius is below 1
// and returns an upper bound on the radius (the largest over strong
// components, each bounded by Collatz ratios of power iteration on A + I).
static double check_attenuation(const Graph& g, const SparseOp& op, double t, const char* name,
                                size_t max_iter) {
  const size_t n = op.dim();
  const double limit = 1.0 / t;
  Components comp = g.directed ? components(pattern_graph(op), true) : components(g, false);
  const size_t k = comp.count();
  std::vector<size_t> start(k + 1, 0);
  for (uint32_t c : comp.membership) start[c + 1] += 1;
  for (size_t c = 0; c < k; ++c) start[c + 1] += start[c];
  std::vector<uint32_t> members(n);
  std::vector<size_t> cursor(start.begin(), start.end() - 1);
  for (size_t v = 0; v < n; ++v) members[cursor[comp.membership[v]]++] = (uint32_t)v;
  std::vector<uint32_t> index(n, 0xFFFFFFFFu);
  double radius = 0.0;
  for (size_t c = 0; c < k; ++c) {
    std::vector<uint32_t> nodes(members.begin() + start[c], members.begin() + start[c + 1]);
    if (nodes.size() == 1) {
      const size_t v = nodes[0];
      double diag = 0.0;
      for (uint64_t q = op.off[v]; q < op.off[v + 1]; ++q)
        if (op.cols[q] == v) diag += op.has_vals ? op.vals[q] : 1.0;
      if (diag >= limit) throw too_large(name, t, diag);
      radius = std::max(radius, diag);
      continue;
    }
    for (size_t i = 0; i < nodes.size(); ++i) index[nodes[i]] = (uint32_t)i;
    SparseOp sub = op.submatrix(nodes, index);
    for (uint32_t v : nodes) index[v] = 0xFFFFFFFFu;
    const size_t m = sub.dim();
    std::vector<double> x(m, 1.0), y(m, 0.0);
    bool decided = false;
    for (size_t it = 0; it < max_iter; ++it) {
      sub.apply(x.data(), y.data());
      double lo = std::numeric_limits<double>::infinity(), hi = 0.0, top = 0.0;
      for (size_t i = 0; i < m; ++i) {
        const double r = y[i] / x[i];
        lo = std::fmin(lo, r);
        hi = std::fmax(hi, r);
        y[i] += x[i];
        top = std::fmax(top, y[i]);
      }
      if (lo >= limit) throw too_large(name, t, lo);
      if (hi < limit) {
        radius = std::max(radius, hi);
        decided = true;
        break;
      }
      for (size_t i = 0; i < m; ++i) x[i] = y[i] / top;
    }
    if (!decided)
      throw Error{std::string(name) + " = " + fmt_g(t) +
                  " is too close to 1 / lambda_max to decide whether the series converges; "
                  "choose a smaller value"};
  }
  return radius;
}

// spectral.rs:346-363: a constant or per-node vector.
static std::vector<double> per_node(const std::vector<double>& v, size_t n, const char* what) {
  std::vector<double> out;
  if (v.size() == 1) out.assign(n, v[0]);
  else if (v.size() == n) out = v;
  else
    throw Error{std::string(what) + ": expected length " + std::to_string(n) + ", found " +
                std::to_string(v.size())};
  for (double x : out)
    if (!std::isfinite(x)) throw Error{std::string(what) + " must be finite"};
  return out;
}

// spectral.rs:365-407.
std::vector<double> katz(const Graph& g, const KatzOptions& o, size_t* iters) {
  check_iteration(o.tol, o.max_iter);
  const size_t n = g.n;
  *iters = 0;
  if (!std::isfinite(o.alpha) || o.alpha < 0.0)
    throw Error{"alpha is " + fmt_g(o.alpha) +
                "; it must be a nonnegative number below 1 / lambda_max"};
  std::vector<double> beta = per_node(o.beta, n, "beta");
  if (n == 0) return {};
  if (o.weighted) check_nonnegative(g, "Katz centrality");
  Graph holder;
  SparseOp op = matrix(g, o.mode, o.weighted, o.loops, o.threads, &holder);
  const double q = o.alpha > 0.0 ? o.alpha * check_attenuation(g, op, o.alpha, "alpha", o.max_iter)
                                 : 0.0;
  std::vector<double> x = solve_series(op, beta, o.alpha, q, o.tol, o.max_iter,
                                       "Katz centrality", iters);
  if (o.normalized) {
    double ss = 0.0;
    for (double v : x) ss += v * v;
    const double norm = std::sqrt(ss);
    if (norm > 0.0)
      for (double& v : x) v /= norm;
  }
  return x;
}

// linalg.rs:357-384 and 433-467.
bool dense_solve_rowmajor(std::vector<double> a, size_t n, std::vector<double>* xio, double tol) {
  std::vector<double>& x = *xio;
  double mag = 0.0;
  for (double v : a) mag = std::max(mag, std::fabs(v));
  mag = std::max(mag, std::numeric_limits<double>::min());
  const double threshold = tol * mag;
  for (size_t k = 0; k < n; ++k) {
    size_t p = k;
    for (size_t r = k + 1; r < n; ++r)
      if (std::fabs(a[r * n + k]) > std::fabs(a[p * n + k])) p = r;
    if (std::fabs(a[p * n + k]) <= threshold) return false;
    if (p != k) {
      for (size_t c = 0; c < n; ++c) std::swap(a[k * n + c], a[p * n + c]);
      std::swap(x[k], x[p]);
    }
    const double pivot = a[k * n + k];
    for (size_t i = k + 1; i < n; ++i) {
      const double f = a[i * n + k] / pivot;
      if (f == 0.0) continue;
      a[i * n + k] = 0.0;
      for (size_t j = k + 1; j < n; ++j) a[i * n + j] = a[i * n + j] - f * a[k * n + j];
      x[i] -= f * x[k];
    }
  }
  for (size_t k = n; k-- > 0;) {
    double s = x[k];
    for (size_t j = k + 1; j < n; ++j) s -= a[k * n + j] * x[j];
    x[k] = s / a[k * n + k];
  }
  return true;
}

// spectral.rs:590-655 (DENSE_MAX 5000) and 657-672.
std::vector<double> bonacich_power(const Graph& g, const BonacichOptions& o, size_t* iters,
                                   bool* dense) {
  check_iteration(o.tol, o.max_iter);
  *iters = 0;
  *dense = false;
  if (!std::isfinite(o.exponent)) throw Error{"the exponent must be finite"};
  const size_t n = g.n;
  if (n == 0) return {};
  if (o.weighted) check_nonnegative(g, "power centrality");
  Graph holder;
  SparseOp op = matrix(g, o.mode, o.weighted, o.loops, o.threads, &holder);
  std::vector<double> ones(n, 1.0), b(n, 0.0);
  op.apply(ones.data(), b.data());
  const double beta = o.exponent;
  bool series = true;
  double q = 0.0;
  if (beta != 0.0) {
    try {
      q = check_attenuation(g, op, std::fabs(beta), "|exponent|", o.max_iter) * std::fabs(beta);
    } catch (const Error&) {
      series = false;
    }
  }
  std::vector<double> y;
  if (series) {
    y = solve_series(op, b, beta, q, o.tol, o.max_iter, "power centrality", iters);
  } else {
    if (n > 5000)
      throw Error{"|exponent| x lambda_max >= 1, so power centrality needs a dense linear "
                  "solve, which is limited to 5000 nodes; use a smaller |exponent|"};
    std::vector<double> a(n * n, 0.0);
    for (size_t i = 0; i < n; ++i) a[i * n + i] = 1.0;
    for (size_t i = 0; i < n; ++i)
      for (uint64_t k = op.off[i]; k < op.off[i + 1]; ++k) {
        const size_t j = op.cols[k];
        a[i * n + j] = a[i * n + j] - beta * (op.has_vals ? op.vals[k] : 1.0);
      }
    y = b;
    if (!dense_solve_rowmajor(a, n, &y, 1e-12))
      throw Error{"I - exponent x A is singular (exponent is the reciprocal of an eigenvalue), "
                  "so power centrality is undefined; choose another exponent"};
    *dense = true;
  }
  double sq = 0.0;
  for (double v : y) sq += v * v;
  const double alpha = std::sqrt((double)n / sq);
  if (o.rescale) {
    double total = 0.0;
    for (double v : y) total += v;
    for (double& v : y) v /= total;
  } else {
    for (double& v : y) v *= alpha;
  }
  return y;
}

// ======================================================== HITS
// SparseOp::transpose (eigenvector.rs:627-656): a stable counting sort by
// column, so row j lists the rows holding column j in increasing order.
static SparseOp transpose_op(const SparseOp& a, size_t ncol) {
  SparseOp t;
  t.has_vals = a.has_vals;
  t.threads = a.threads;
  t.off.assign(ncol + 1, 0);
  for (uint32_t j : a.cols) t.off[j + 1] += 1;
  for (size_t c = 0; c < ncol; ++c) t.off[c + 1] += t.off[c];
  std::vector<uint64_t> cur(t.off.begin(), t.off.end() - 1);
  t.cols.assign(a.cols.size(), 0);
  if (a.has_vals) t.vals.assign(a.cols.size(), 0.0);
  for (size_t v = 0; v < a.dim(); ++v)
    for (uint64_t k = a.off[v]; k < a.off[v + 1]; ++k) {
      const uint64_t slot = cur[a.cols[k]]++;
      t.cols[slot] = (uint32_t)v;
      if (a.has_vals) t.vals[slot] = a.vals[k];
    }
  return t;
}

static double entry(const SparseOp& a, uint64_t k) { return a.has_vals ? a.vals[k] : 1.0; }

// spectral.rs:905-922: sum of squares of row v, parallel entries merged.
static double merged_squares(const SparseOp& a, size_t v) {
  double q = 0.0, acc = 0.0;
  bool open = false;
  uint32_t c = 0;
  for (uint64_t k = a.off[v]; k < a.off[v + 1]; ++k) {
    if (open && a.cols[k] == c) {
      acc += entry(a, k);
    } else {
      if (open) q += acc * acc;
      c = a.cols[k];
      acc = entry(a, k);
      open = true;
    }
  }
  if (open) q += acc * acc;
  return q;
}

// spectral.rs:924-938.
static void hits_rescale(std::vector<double>& x, int how) {
  for (double& v : x)
    if (v < 0.0) v = 0.0;
  double d = 0.0;
  if (how == 0) {
    for (double v : x) d = std::max(d, v);
  } else if (how == 1) {
    for (double v : x) d += v;
  } else {
    for (double v : x) d += v * v;
    d = std::sqrt(d);
  }
  if (d > 0.0)
    for (double& v : x) v /= d;
}

// spectral.rs:748-903.
Hits hits(const Graph& g, const HitsOptions& o) {
  check_iteration(o.tol, o.max_iter);
  const size_t n = g.n;
  if (o.weighted) check_nonnegative(g, "hub and authority scores");
  Graph holder;
  SparseOp a = matrix(g, Mode::Out, o.weighted, o.loops, o.threads, &holder);
  SparseOp at = transpose_op(a, n);
  // blocks of the bipartite graph (hubs 0..n, authorities n..2n)
  std::vector<size_t> parent(2 * n);
  std::iota(parent.begin(), parent.end(), 0);
  std::function<size_t(size_t)> find = [&](size_t v) {
    while (parent[v] != v) {
      parent[v] = parent[parent[v]];
      v = parent[v];
    }
    return v;
  };
  bool any = false;
  for (size_t i = 0; i < n; ++i)
    for (uint64_t k = a.off[i]; k < a.off[i + 1]; ++k)
      if (entry(a, k) > 0.0) {
        any = true;
        size_t x = find(i), y = find(n + a.cols[k]);
        if (x != y) parent[std::max(x, y)] = std::min(x, y);
      }
  Hits r;
  if (!any) {
    r.hubs.assign(n, std::numeric_limits<double>::quiet_NaN());
    r.authorities.assign(n, std::numeric_limits<double>::quiet_NaN());
    r.value = 0.0;
    r.unique = false;
    return r;
  }
  std::vector<char> has_in(n, 0), has_out(n, 0);
  for (size_t j = 0; j < n; ++j)
    for (uint64_t k = at.off[j]; k < at.off[j + 1]; ++k)
      if (entry(at, k) > 0.0) has_in[j] = 1;
  for (size_t i = 0; i < n; ++i)
    for (uint64_t k = a.off[i]; k < a.off[i + 1]; ++k)
      if (entry(a, k) > 0.0) has_out[i] = 1;
  std::vector<size_t> block_of(2 * n, SIZE_MAX);
  std::vector<std::vector<uint32_t>> bh, ba;
  for (size_t v = 0; v < 2 * n; ++v) {
    const bool present = v < n ? has_out[v] : has_in[v - n];
    if (!present) continue;
    const size_t root = find(v);
    if (block_of[root] == SIZE_MAX) {
      block_of[root] = bh.size();
      bh.emplace_back();
      ba.emplace_back();
    }
    if (v < n) bh[block_of[root]].push_back((uint32_t)v);
    else ba[block_of[root]].push_back((uint32_t)(v - n));
  }
  std::vector<double> row_sum(n, 0.0), col_sum(n, 0.0), col_sq(n, 0.0);
  for (size_t i = 0; i < n; ++i)
    for (uint64_t k = a.off[i]; k < a.off[i + 1]; ++k) row_sum[i] += entry(a, k);
  for (size_t j = 0; j < n; ++j) {
    for (uint64_t k = at.off[j]; k < at.off[j + 1]; ++k) col_sum[j] += entry(at, k);
    col_sq[j] = merged_squares(at, j);
  }
  const size_t kb = bh.size();
  std::vector<double> upper(kb, 0.0), lower(kb, 0.0);
  for (size_t b = 0; b < kb; ++b) {
    double rmax = 0.0, cmax = 0.0, lmax = 0.0;
    for (uint32_t i : bh[b]) rmax = std::max(rmax, row_sum[i]);
    for (uint32_t j : ba[b]) {
      cmax = std::max(cmax, col_sum[j]);
      lmax = std::max(lmax, col_sq[j]);
    }
    upper[b] = rmax * cmax;
    lower[b] = lmax;
  }
  std::vector<size_t> order(kb);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(),
                   [&](size_t x, size_t y) { return lower[x] > lower[y]; });
  std::vector<uint32_t> hub_index(n, 0xFFFFFFFFu), auth_index(n, 0xFFFFFFFFu);
  double best = 0.0;
  struct Solved {
    size_t b;
    double value;
    std::vector<double> v, s;
  };
  std::vector<Solved> solved;
  for (size_t b : order) {
    if (upper[b] < best * (1.0 - TIE)) continue;
    for (size_t i = 0; i < bh[b].size(); ++i) hub_index[bh[b][i]] = (uint32_t)i;
    for (size_t i = 0; i < ba[b].size(); ++i) auth_index[ba[b][i]] = (uint32_t)i;
    SparseOp ab = a.submatrix(bh[b], auth_index);
    SparseOp abt = at.submatrix(ba[b], hub_index);
    for (uint32_t v : bh[b]) hub_index[v] = 0xFFFFFFFFu;
    for (uint32_t v : ba[b]) auth_index[v] = 0xFFFFFFFFu;
    std::vector<double> ones(bh[b].size(), 1.0), sv(ba[b].size(), 0.0);
    abt.apply(ones.data(), sv.data());
    std::vector<double> tmp(ab.dim(), 0.0);
    Leading res;
    if (!symmetric_leading(ba[b].size(),
                           [&](const double* x, double* y) {
                             ab.apply(x, tmp.data());
                             abt.apply(tmp.data(), y);
                           },
                           sv, o.tol, 0.0, o.max_iter, &res))
      throw Error{"hub and authority scores did not converge to tolerance " + fmt_g(o.tol) +
                  " within " + std::to_string(o.max_iter) +
                  " matrix-vector products; a larger iteration cap may help"};
    best = std::max(best, res.value);
    solved.push_back({b, res.value, std::move(res.vector), std::move(sv)});
  }
  std::vector<double> auth(n, 0.0);
  size_t tied = 0;
  for (const Solved& sv : solved) {
    if (sv.value < best * (1.0 - TIE)) continue;
    ++tied;
    double weight = 0.0;
    for (size_t i = 0; i < sv.v.size(); ++i) weight += sv.v[i] * sv.s[i];
    for (size_t i = 0; i < ba[sv.b].size(); ++i) auth[ba[sv.b][i]] = sv.v[i] * weight;
  }
  std::vector<double> hubs(n, 0.0);
  a.apply(auth.data(), hubs.data());
  hits_rescale(auth, o.scale);
  hits_rescale(hubs, o.scale);
  r.hubs = std::move(hubs);
  r.authorities = std::move(auth);
  r.value = best;
  r.unique = tied == 1;
  return r;
}

// ======================================================== G(n, m)
// generate.rs:148-155.
static uint64_t pair_count(uint64_t n, bool directed, bool loops) {
  if (directed) return loops ? n * n : n * (n ? n - 1 : 0);
  return loops ? n * (n + 1) / 2 : n * (n ? n - 1 : 0) / 2;
}

static uint64_t isqrt(uint64_t x) {
  uint64_t r = (uint64_t)std::sqrt((double)x);
  while (r > 0 && r * r > x) --r;
  while ((r + 1) * (r + 1) <= x) ++r;
  return r;
}

// generate.rs:169-205: the k-th candidate pair.
static void decode(uint64_t k, uint64_t n, bool directed, bool loops, uint64_t* a, uint64_t* b) {
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

// generate.rs:255-290: Floyd's sampling of m distinct candidate indices,
// decoded and sorted by (from, to).
void gnm(size_t n, uint64_t m, bool directed, bool loops, uint64_t seed, uint64_t rep,
         std::vector<uint32_t>* from, std::vector<uint32_t>* to) {
  Stream rng(seed, rep);
  uint64_t total = pair_count(n, directed, loops);
  if (m > total) throw Error{"too many edges for G(n, m)"};
  std::vector<uint64_t> chosen;
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
  std::sort(chosen.begin(), chosen.end());
  std::vector<std::pair<uint32_t, uint32_t>> pairs;
  pairs.reserve(chosen.size());
  for (uint64_t k : chosen) {
    uint64_t a, b;
    decode(k, n, directed, loops, &a, &b);
    pairs.push_back({(uint32_t)a, (uint32_t)b});
  }
  std::sort(pairs.begin(), pairs.end());
  from->resize(pairs.size());
  to->resize(pairs.size());
  for (size_t i = 0; i < pairs.size(); ++i) {
    (*from)[i] = pairs[i].first;
    (*to)[i] = pairs[i].second;
  }
}

}  // namespace orc
