// C entry points of the CPU oracle: TEST INFRASTRUCTURE ONLY.
//
// They mirror the reference's C ABI (crates/capi/include/netcapi.h) with an
// `orc_` prefix so that the parity tests call the oracle and the product
// library with identical arguments. Status 0 is success; on failure 1 is
// returned and a message is written to err (crates/capi/src/lib.rs:57-87).
#include <chrono>
#include <cmath>
#include <cstring>
#include <exception>
#include <thread>
#include <vector>

#include "oracle.hpp"

using namespace orc;

struct OrcGraph {
  Graph g;
};

static void write_err(char* err, size_t len, const std::string& msg) {
  if (!err || len == 0) return;
  size_t k = std::min(msg.size(), len - 1);
  memcpy(err, msg.data(), k);
  err[k] = 0;
}

template <class F>
static int32_t guard(char* err, size_t len, F f) {
  try {
    f();
    return 0;
  } catch (const Error& e) {
    write_err(err, len, e.msg);
  } catch (const std::exception& e) {
    write_err(err, len, std::string("internal error in the oracle: ") + e.what());
  }
  return 1;
}

static const Graph& handle(const OrcGraph* h) {
  if (!h) throw Error{"graph handle is null"};
  return h->g;
}

// Runs f(lo, hi) over [0, count) in contiguous blocks on every host core;
// every element depends on its own index only, so results do not depend on
// the thread count.
template <class F>
static void for_blocks(int64_t count, F f) {
  const int64_t nt = std::max<int64_t>(
      1, std::min<int64_t>(std::thread::hardware_concurrency(), (count + 65535) / 65536));
  std::vector<std::thread> pool;
  for (int64_t t = 0; t < nt; ++t)
    pool.emplace_back([&, t] { f(count * t / nt, count * (t + 1) / nt); });
  for (auto& th : pool) th.join();
}

extern "C" {

void orc_philox4x32_10(const uint32_t* ctr, const uint32_t* key, uint32_t* out) {
  philox4x32_10(ctr, key, out);
}

void orc_stream_u32(uint64_t seed, uint64_t index, int64_t count, uint32_t* out) {
  Stream s(seed, index);
  for (int64_t i = 0; i < count; ++i) out[i] = s.next_u32();
}

void orc_stream_below(uint64_t seed, uint64_t index, uint64_t bound, int64_t count, uint64_t* out) {
  Stream s(seed, index);
  for (int64_t i = 0; i < count; ++i) out[i] = s.below(bound);
}

int32_t orc_gnm(int64_t n, int64_t m, int32_t directed, int32_t loops, uint64_t seed, uint64_t rep,
                uint32_t* from, uint32_t* to, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    std::vector<uint32_t> f, t;
    gnm((size_t)n, (uint64_t)m, directed != 0, loops != 0, seed, rep, &f, &t);
    memcpy(from, f.data(), f.size() * 4);
    memcpy(to, t.data(), t.size() * 4);
  });
}

// R-MAT edges (Chakrabarti, Zhan and Faloutsos 2004) as defined by this
// project: edge k draws `scale` 32-bit words from stream (seed, k), most
// significant level first, and picks quadrant a / b / c / d by comparing a
// word with floor(a 2^32), floor((a+b) 2^32), floor((a+b+c) 2^32).
void orc_rmat(int32_t scale, int64_t m, double a, double b, double c, uint64_t seed,
              uint32_t* src, uint32_t* tgt) {
  const double two32 = 4294967296.0;
  uint64_t ta = (uint64_t)(a * two32), tab = (uint64_t)((a + b) * two32),
           tabc = (uint64_t)((a + b + c) * two32);
  for_blocks(m, [&](int64_t lo, int64_t hi) {
    for (int64_t k = lo; k < hi; ++k) {
      Stream s(seed, (uint64_t)k);
      uint32_t r = 0, q = 0;
      for (int l = 0; l < scale; ++l) {
        uint64_t u = s.next_u32();
        uint32_t rb = u >= tab ? 1u : 0u;
        uint32_t cb = (u >= ta && u < tab) || u >= tabc ? 1u : 0u;
        r = r << 1 | rb;
        q = q << 1 | cb;
      }
      src[k] = r;
      tgt[k] = q;
    }
  });
}

// Lognormal(0, 1) strengths rounded to FP32, as this project defines them:
// for edge e the first four words of stream (seed, e) make two 53-bit
// uniforms u1, u2 in [0, 1), and w = exp(sqrt(-2 ln(1 - u1)) cos(2 pi u2))
// (Box and Muller 1958).
void orc_lognormal(int64_t m, uint64_t seed, float* w) {
  for_blocks(m, [&](int64_t lo, int64_t hi) {
    for (int64_t e = lo; e < hi; ++e) {
      Stream s(seed, (uint64_t)e);
      uint64_t r0 = s.next_u32(), r1 = s.next_u32(), r2 = s.next_u32(), r3 = s.next_u32();
      const uint64_t a = (r0 << 32 | r1) >> 11, b = (r2 << 32 | r3) >> 11;
      const double u1 = (double)a / 9007199254740992.0, u2 = (double)b / 9007199254740992.0;
      const double z = std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(6.283185307179586 * u2);
      w[e] = (float)std::exp(z);
    }
  });
}

int32_t orc_graph_new(int64_t n, const int64_t* src, const int64_t* tgt, const double* weights,
                      int64_t m, int32_t directed, OrcGraph** out, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    if (n < 0 || m < 0) throw Error{"negative node or edge count"};
    auto* h = new OrcGraph;
    try {
      h->g = graph_from_edges((size_t)n, src, tgt, weights, (size_t)m, directed != 0);
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

void orc_graph_free(OrcGraph* h) { delete h; }

int64_t orc_graph_node_count(const OrcGraph* h) { return h ? (int64_t)h->g.n : -1; }
int64_t orc_graph_edge_count(const OrcGraph* h) { return h ? (int64_t)h->g.src.size() : -1; }
int64_t orc_graph_arc_count(const OrcGraph* h, int32_t which) {
  if (!h) return -1;
  return (int64_t)(which == 1 ? h->g.in_rows().arcs() : h->g.out.arcs());
}

// CSR arrays of the out (which = 0) or in (which = 1) adjacency.
void orc_graph_csr(const OrcGraph* h, int32_t which, uint64_t* off, uint32_t* tgt, double* w) {
  const Csr& c = which == 1 ? h->g.in_rows() : h->g.out;
  memcpy(off, c.off.data(), c.off.size() * 8);
  memcpy(tgt, c.tgt.data(), c.tgt.size() * 4);
  if (w && c.weighted) memcpy(w, c.w.data(), c.w.size() * 8);
}

int32_t orc_degree(const OrcGraph* h, int32_t mode, int32_t loops, int32_t weighted, double* out,
                   char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    const Graph& g = handle(h);
    auto v = degree(g, mode_from_code(mode), loops != 0, weighted != 0);
    memcpy(out, v.data(), v.size() * 8);
  });
}

int32_t orc_components(const OrcGraph* h, int32_t strong, uint32_t* membership, int64_t* count) {
  Components c = components(h->g, strong != 0);
  memcpy(membership, c.membership.data(), c.membership.size() * 4);
  *count = (int64_t)c.count();
  return 0;
}

// net_pagerank (crates/capi/src/spectral.rs:59-97) plus the iteration count
// and, for CPU timing only, a fixed number of iterations (fixed_iters > 0).
int32_t orc_pagerank_ex(const OrcGraph* h, double damping, int32_t directed, int32_t weighted,
                        const double* personalization, int32_t dangling, int32_t loops, double tol,
                        int64_t max_iter, int32_t threads, int64_t fixed_iters, double* out,
                        int64_t* iters, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    const Graph& g = handle(h);
    PagerankOptions o;
    o.damping = damping;
    o.directed = directed != 0;
    o.weighted = weighted != 0;
    o.personalization = personalization;
    if (dangling != 0 && dangling != 1)
      throw Error{"unknown dangling-node code " + std::to_string(dangling)};
    o.dangling = dangling;
    o.loops = loops_from_code(loops);
    o.tol = tol > 0 ? tol : 1e-12;
    o.max_iter = max_iter > 0 ? (size_t)max_iter : 10000;
    o.threads = threads > 0 ? (size_t)threads : 0;
    o.fixed_iters = fixed_iters > 0 ? (size_t)fixed_iters : 0;
    size_t it = 0;
    auto v = pagerank(g, o, &it);
    if (!v.empty()) memcpy(out, v.data(), v.size() * 8);
    if (iters) *iters = (int64_t)it;
  });
}

int32_t orc_pagerank(const OrcGraph* h, double damping, int32_t directed, int32_t weighted,
                     const double* personalization, int32_t dangling, int32_t loops, double tol,
                     int64_t max_iter, int32_t threads, double* out, char* err, size_t err_len) {
  return orc_pagerank_ex(h, damping, directed, weighted, personalization, dangling, loops, tol,
                         max_iter, threads, 0, out, nullptr, err, err_len);
}

// The PageRank iteration on a prebuilt pull operator (rows = arcs arriving
// at a node, with out-strength `out_strength`), uniform teleport. Times
// exactly `fixed_iters` iterations with `threads` threads and returns the
// seconds spent; the CPU-baseline leg of the benchmark uses it.
double orc_pagerank_time_op(int64_t n, const uint64_t* off, const uint32_t* cols,
                            const double* vals, const double* out_strength, double damping,
                            int64_t fixed_iters, int32_t threads, double* out) {
  SparseOp op;
  op.off.assign(off, off + n + 1);
  op.cols.assign(cols, cols + off[n]);
  op.has_vals = vals != nullptr;
  if (vals) op.vals.assign(vals, vals + off[n]);
  op.threads = threads_for(threads > 0 ? threads : 0, (size_t)n, off[n] / 2);
  std::vector<double> os(out_strength, out_strength + n);
  std::vector<double> p((size_t)n, 1.0 / (double)n);
  size_t it = 0;
  auto t0 = std::chrono::steady_clock::now();
  auto x = pagerank_on_op(op, os, damping, p, p, 1e-300, (size_t)fixed_iters, (size_t)fixed_iters,
                          &it);
  auto t1 = std::chrono::steady_clock::now();
  if (out) memcpy(out, x.data(), x.size() * 8);
  return std::chrono::duration<double>(t1 - t0).count();
}

int64_t orc_threads_for(int32_t requested, int64_t items, int64_t work) {
  return (int64_t)threads_for(requested > 0 ? requested : 0, (size_t)items, (uint64_t)work);
}

// net_eigenvector (crates/capi/src/topography.rs:208-249) plus the count
// of matrix-vector products.
int32_t orc_eigenvector_ex(const OrcGraph* h, int32_t mode, int32_t weighted, int32_t scale,
                           int32_t loops, double tol, int64_t max_iter, int32_t threads,
                           double* out, double* eigenvalue, int32_t* connected, int64_t* iters,
                           char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    const Graph& g = handle(h);
    EigenvectorOptions o;
    o.mode = mode_from_code(mode);
    o.weighted = weighted != 0;
    if (scale != 0 && scale != 1)
      throw Error{"unknown eigenvector scale code " + std::to_string(scale)};
    o.scale = scale;
    o.loops = loops_from_code(loops);
    o.tol = tol > 0 ? tol : 1e-12;
    o.max_iter = max_iter > 0 ? (size_t)max_iter : 10000;
    o.threads = threads > 0 ? (size_t)threads : 0;
    Eigenvector e = eigenvector_centrality(g, o);
    if (!e.values.empty()) memcpy(out, e.values.data(), e.values.size() * 8);
    *eigenvalue = e.eigenvalue;
    *connected = e.connected ? 1 : 0;
    if (iters) *iters = (int64_t)e.iterations;
  });
}

int32_t orc_eigenvector(const OrcGraph* h, int32_t mode, int32_t weighted, int32_t scale,
                        int32_t loops, double tol, int64_t max_iter, int32_t threads, double* out,
                        double* eigenvalue, int32_t* connected, char* err, size_t err_len) {
  return orc_eigenvector_ex(h, mode, weighted, scale, loops, tol, max_iter, threads, out,
                            eigenvalue, connected, nullptr, err, err_len);
}

// net_katz / net_bonacich_power (crates/capi/src/spectral.rs:107-179), plus
// the iteration count and (Bonacich) whether the dense solve was used.
int32_t orc_katz(const OrcGraph* h, double alpha, const double* beta, int64_t beta_len,
                 int32_t mode, int32_t weighted, int32_t loops, int32_t normalized, double tol,
                 int64_t max_iter, int32_t threads, double* out, int64_t* iters, char* err,
                 size_t err_len) {
  return guard(err, err_len, [&] {
    const Graph& g = handle(h);
    if (beta_len < 0) throw Error{"beta length must be nonnegative"};
    KatzOptions o;
    o.alpha = alpha;
    o.beta.assign(beta, beta + beta_len);
    o.mode = mode_from_code(mode);
    o.weighted = weighted != 0;
    o.loops = loops_from_code(loops);
    o.normalized = normalized != 0;
    o.tol = tol > 0 ? tol : 1e-12;
    o.max_iter = max_iter > 0 ? (size_t)max_iter : 10000;
    o.threads = threads > 0 ? (size_t)threads : 0;
    size_t it = 0;
    std::vector<double> x = katz(g, o, &it);
    if (!x.empty()) memcpy(out, x.data(), x.size() * 8);
    if (iters) *iters = (int64_t)it;
  });
}

int32_t orc_bonacich_power(const OrcGraph* h, double exponent, int32_t mode, int32_t weighted,
                           int32_t loops, int32_t rescale, double tol, int64_t max_iter,
                           int32_t threads, double* out, int64_t* iters, int32_t* dense,
                           char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    const Graph& g = handle(h);
    BonacichOptions o;
    o.exponent = exponent;
    o.mode = mode_from_code(mode);
    o.weighted = weighted != 0;
    o.loops = loops_from_code(loops);
    o.rescale = rescale != 0;
    o.tol = tol > 0 ? tol : 1e-12;
    o.max_iter = max_iter > 0 ? (size_t)max_iter : 10000;
    o.threads = threads > 0 ? (size_t)threads : 0;
    size_t it = 0;
    bool dn = false;
    std::vector<double> x = bonacich_power(g, o, &it, &dn);
    if (!x.empty()) memcpy(out, x.data(), x.size() * 8);
    if (iters) *iters = (int64_t)it;
    if (dense) *dense = dn ? 1 : 0;
  });
}

// net_hits (crates/capi/src/spectral.rs:189-230).
int32_t orc_hits(const OrcGraph* h, int32_t weighted, int32_t loops, int32_t scale, double tol,
                 int64_t max_iter, int32_t threads, double* hubs, double* auths, double* value,
                 int32_t* unique, char* err, size_t err_len) {
  return guard(err, err_len, [&] {
    const Graph& g = handle(h);
    HitsOptions o;
    o.weighted = weighted != 0;
    o.loops = loops_from_code(loops);
    if (scale < 0 || scale > 2)
      throw Error{"unknown hub and authority scale code " + std::to_string(scale)};
    o.scale = scale;
    o.tol = tol > 0 ? tol : 1e-12;
    o.max_iter = max_iter > 0 ? (size_t)max_iter : 10000;
    o.threads = threads > 0 ? (size_t)threads : 0;
    Hits r = hits(g, o);
    if (!r.hubs.empty()) memcpy(hubs, r.hubs.data(), r.hubs.size() * 8);
    if (!r.authorities.empty()) memcpy(auths, r.authorities.data(), r.authorities.size() * 8);
    *value = r.value;
    *unique = r.unique ? 1 : 0;
  });
}

// Eigenvalues ascending and eigenvectors (columns of the row-major n x n
// `vecs`) of the symmetric matrix `a`; 1 if the QL iteration fails.
int32_t orc_symmetric_eigen(int64_t n, const double* a, double* vals, double* vecs) {
  std::vector<double> A(a, a + n * n), v, V;
  if (!symmetric_eigen(A, (size_t)n, &v, &V)) return 1;
  memcpy(vals, v.data(), n * 8);
  memcpy(vecs, V.data(), n * n * 8);
  return 0;
}

}  // extern "C"
