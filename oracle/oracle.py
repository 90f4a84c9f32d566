"""ctypes wrapper of the CPU oracle (oracle/liboracle.so): TEST INFRASTRUCTURE ONLY.

The oracle restates the reference engine's spectral-centrality path in C++
(see oracle.hpp). Tests, the smoke check and the benchmark's CPU-baseline leg
use it as the checker; the product library never imports it.
"""
from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
ERR_LEN = 1024

_lib = None


class OracleError(RuntimeError):
    pass


def build(force: bool = False) -> Path:
    """Compiles the oracle with its Makefile (g++)."""
    if force or not LIB_PATH.exists():
        subprocess.run(["make", "-C", str(HERE)] + (["-B"] if force else []), check=True,
                       capture_output=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    build()
    L = ctypes.CDLL(str(LIB_PATH))
    i32, i64, u64, f64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double
    vp, cp, sz = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t
    L.orc_philox4x32_10.argtypes = [vp, vp, vp]
    L.orc_stream_u32.argtypes = [u64, u64, i64, vp]
    L.orc_stream_below.argtypes = [u64, u64, u64, i64, vp]
    L.orc_gnm.argtypes = [i64, i64, i32, i32, u64, u64, vp, vp, cp, sz]
    L.orc_gnm.restype = i32
    L.orc_rmat.argtypes = [i32, i64, f64, f64, f64, u64, vp, vp]
    L.orc_lognormal.argtypes = [i64, u64, vp]
    L.orc_graph_new.argtypes = [i64, vp, vp, vp, i64, i32, ctypes.POINTER(vp), cp, sz]
    L.orc_graph_new.restype = i32
    L.orc_graph_free.argtypes = [vp]
    L.orc_graph_node_count.argtypes = [vp]
    L.orc_graph_node_count.restype = i64
    L.orc_graph_edge_count.argtypes = [vp]
    L.orc_graph_edge_count.restype = i64
    L.orc_graph_arc_count.argtypes = [vp, i32]
    L.orc_graph_arc_count.restype = i64
    L.orc_graph_csr.argtypes = [vp, i32, vp, vp, vp]
    L.orc_degree.argtypes = [vp, i32, i32, i32, vp, cp, sz]
    L.orc_degree.restype = i32
    L.orc_components.argtypes = [vp, i32, vp, ctypes.POINTER(i64)]
    L.orc_components.restype = i32
    L.orc_pagerank_ex.argtypes = [vp, f64, i32, i32, vp, i32, i32, f64, i64, i32, i64, vp,
                                  ctypes.POINTER(i64), cp, sz]
    L.orc_pagerank_ex.restype = i32
    L.orc_pagerank_time_op.argtypes = [i64, vp, vp, vp, vp, f64, i64, i32, vp]
    L.orc_pagerank_time_op.restype = f64
    L.orc_threads_for.argtypes = [i32, i64, i64]
    L.orc_threads_for.restype = i64
    L.orc_eigenvector_ex.argtypes = [vp, i32, i32, i32, i32, f64, i64, i32, vp,
                                     ctypes.POINTER(f64), ctypes.POINTER(i32),
                                     ctypes.POINTER(i64), cp, sz]
    L.orc_eigenvector_ex.restype = i32
    L.orc_symmetric_eigen.argtypes = [i64, vp, vp, vp]
    L.orc_symmetric_eigen.restype = i32
    L.orc_katz.argtypes = [vp, f64, vp, i64, i32, i32, i32, i32, f64, i64, i32, vp,
                           ctypes.POINTER(i64), cp, sz]
    L.orc_katz.restype = i32
    L.orc_bonacich_power.argtypes = [vp, f64, i32, i32, i32, i32, f64, i64, i32, vp,
                                     ctypes.POINTER(i64), ctypes.POINTER(i32), cp, sz]
    L.orc_bonacich_power.restype = i32
    L.orc_hits.argtypes = [vp, i32, i32, i32, f64, i64, i32, vp, vp, ctypes.POINTER(f64),
                           ctypes.POINTER(i32), cp, sz]
    L.orc_hits.restype = i32
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def philox(ctr, key):
    c = np.asarray(ctr, dtype=np.uint32)
    k = np.asarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().orc_philox4x32_10(_ptr(c), _ptr(k), _ptr(out))
    return out


def stream_u32(seed: int, index: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint32)
    lib().orc_stream_u32(seed, index, count, _ptr(out))
    return out


def stream_below(seed: int, index: int, bound: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint64)
    lib().orc_stream_below(seed, index, bound, count, _ptr(out))
    return out


def gnm(n: int, m: int, directed: bool = False, loops: bool = False, seed: int = 1,
        rep: int = 0):
    f = np.zeros(m, dtype=np.uint32)
    t = np.zeros(m, dtype=np.uint32)
    err = ctypes.create_string_buffer(ERR_LEN)
    if lib().orc_gnm(n, m, int(directed), int(loops), seed, rep, _ptr(f), _ptr(t), err, ERR_LEN):
        raise OracleError(err.value.decode())
    return f, t


def rmat_raw(scale: int, m: int, a: float, b: float, c: float, seed: int):
    s = np.zeros(m, dtype=np.uint32)
    t = np.zeros(m, dtype=np.uint32)
    lib().orc_rmat(scale, m, a, b, c, seed, _ptr(s), _ptr(t))
    return s, t


def rmat(scale: int, edge_factor: int, a: float, b: float, c: float, seed: int,
         clean: bool = True, symmetrize: bool = False):
    """R-MAT edges as the library's generator makes them: raw draws, or with
    self-loops and duplicate arcs removed (edges sorted by (source, target));
    symmetrize keeps each unordered pair once as (smaller, larger)."""
    s, t = rmat_raw(scale, edge_factor << scale, a, b, c, seed)
    if not clean and not symmetrize:
        return s, t
    keep = s != t
    s, t = s[keep].astype(np.int64), t[keep].astype(np.int64)
    if symmetrize:
        s, t = np.minimum(s, t), np.maximum(s, t)
    key = np.sort(s << scale | t)
    if len(key):
        key = key[np.concatenate(([True], key[1:] != key[:-1]))]
    return (key >> scale).astype(np.uint32), (key & ((1 << scale) - 1)).astype(np.uint32)


def lognormal(m: int, seed: int) -> np.ndarray:
    """Lognormal(0, 1) strengths of edges 0 .. m - 1 rounded to FP32, as the
    library's generator draws them (Box-Muller on stream (seed, edge))."""
    w = np.zeros(m, dtype=np.float32)
    lib().orc_lognormal(m, seed, _ptr(w))
    return w


class Graph:
    """An oracle graph handle (mirror of net_graph_new / net_graph_free)."""

    def __init__(self, n, src, tgt, weights=None, directed=True):
        self.n = int(n)
        s = np.ascontiguousarray(src, dtype=np.int64)
        t = np.ascontiguousarray(tgt, dtype=np.int64)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        self.m = len(s)
        self.directed = bool(directed)
        self.weighted = w is not None
        self._src, self._tgt, self._w = s, t, w
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(ERR_LEN)
        if lib().orc_graph_new(self.n, _ptr(s), _ptr(t), _ptr(w), self.m, int(directed),
                               ctypes.byref(h), err, ERR_LEN):
            raise OracleError(err.value.decode())
        self.h = h

    def __del__(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.orc_graph_free(self.h)
            self.h = None

    def csr(self, which: int = 0):
        arcs = lib().orc_graph_arc_count(self.h, which)
        off = np.zeros(self.n + 1, dtype=np.uint64)
        tgt = np.zeros(max(arcs, 1), dtype=np.uint32)
        w = np.zeros(max(arcs, 1), dtype=np.float64) if self.weighted else None
        lib().orc_graph_csr(self.h, which, _ptr(off), _ptr(tgt), _ptr(w))
        return off, tgt[:arcs], (None if w is None else w[:arcs])

    def degree(self, mode=3, loops=True, weighted=False):
        out = np.zeros(max(self.n, 1))
        err = ctypes.create_string_buffer(ERR_LEN)
        if lib().orc_degree(self.h, mode, int(loops), int(weighted), _ptr(out), err, ERR_LEN):
            raise OracleError(err.value.decode())
        return out[: self.n]

    def components(self, strong=False):
        memb = np.zeros(max(self.n, 1), dtype=np.uint32)
        cnt = ctypes.c_int64()
        lib().orc_components(self.h, int(strong), _ptr(memb), ctypes.byref(cnt))
        return memb[: self.n], cnt.value

    def pagerank(self, damping=0.85, directed=True, weighted=False, personalization=None,
                 dangling=0, loops=0, tol=0.0, max_iter=0, threads=0, fixed_iters=0):
        out = np.zeros(max(self.n, 1))
        p = None if personalization is None else np.ascontiguousarray(personalization,
                                                                       dtype=np.float64)
        it = ctypes.c_int64()
        err = ctypes.create_string_buffer(ERR_LEN)
        if lib().orc_pagerank_ex(self.h, damping, int(directed), int(weighted), _ptr(p),
                                 dangling, loops, tol, max_iter, threads, fixed_iters, _ptr(out),
                                 ctypes.byref(it), err, ERR_LEN):
            raise OracleError(err.value.decode())
        self.last_iters = it.value
        return out[: self.n]

    def eigenvector(self, mode=2, weighted=False, scale=0, loops=0, tol=0.0, max_iter=0,
                    threads=0):
        out = np.zeros(max(self.n, 1))
        val = ctypes.c_double()
        conn = ctypes.c_int32()
        it = ctypes.c_int64()
        err = ctypes.create_string_buffer(ERR_LEN)
        if lib().orc_eigenvector_ex(self.h, mode, int(weighted), scale, loops, tol, max_iter,
                                    threads, _ptr(out), ctypes.byref(val), ctypes.byref(conn),
                                    ctypes.byref(it), err, ERR_LEN):
            raise OracleError(err.value.decode())
        self.last_iters = it.value
        return out[: self.n], val.value, bool(conn.value)


    def edges(self):
        return self._src.copy(), self._tgt.copy(), (None if self._w is None else self._w.copy())

    def simplify(self, undirected=False, keep=0):
        """simplify (crates/engine/src/metrics/topography.rs:96-141): loops
        dropped; each arc, or for an undirected result each pair as
        (smaller, larger), once in (from, to) order with the largest (keep 0)
        or smallest (keep 1) weight of its parallel edges."""
        if keep not in (0, 1):
            raise OracleError(f"unknown parallel-edge weight code {keep}")
        directed = self.directed and not undirected
        s, t, w = self._src, self._tgt, self._w
        keepm = s != t
        s, t = s[keepm], t[keepm]
        x = np.ones(len(s)) if w is None else w[keepm]
        if not directed:
            lo, hi = np.minimum(s, t), np.maximum(s, t)
            s, t = lo, hi
        merged = {}
        for a, b, v in zip(s.tolist(), t.tolist(), x.tolist()):
            k = (a, b)
            if k in merged:
                merged[k] = min(merged[k], v) if keep else max(merged[k], v)
            else:
                merged[k] = v
        keys = sorted(merged)
        ms = np.array([k[0] for k in keys], dtype=np.int64)
        mt = np.array([k[1] for k in keys], dtype=np.int64)
        mw = None if w is None else np.array([merged[k] for k in keys])
        return Graph(self.n, ms, mt, mw, directed)

    def twomode_eigenvector(self, types, tol=0.0, max_iter=0):
        """twomode_eigenvector (crates/engine/src/metrics/bipartite.rs:93-111,
        113-116, 288-336; type codes as crates/capi/src/twomode.rs:50-66):
        eigenvector centrality of the binary affiliation graph (undirected,
        parallel edges merged), direction ignored, unweighted, unit scale,
        loops ignored; each mode's half divided by its own Euclidean norm
        (a sequential sum in node order); NaN everywhere without ties."""
        types = [int(v) for v in types]
        for v, c in enumerate(types):
            if c not in (0, 1):
                raise OracleError(f"node {v} has type code {c}; use 0 for the first mode "
                                  "and 1 for the second")
        for e, (a, b) in enumerate(zip(self._src.tolist(), self._tgt.tolist())):
            if types[a] == types[b]:
                raise OracleError(f"edge {e} joins nodes {a} and {b}, which are in the same "
                                  "mode; in a two-mode network every edge joins the two modes")
        aff = self.simplify(undirected=True, keep=0)
        x, lam, conn = aff.eigenvector(mode=3, weighted=False, scale=1, loops=2, tol=tol,
                                       max_iter=max_iter)
        if aff.m == 0:
            return np.full(self.n, np.nan), 0.0, conn
        x = x.copy()
        for mode in (0, 1):
            ss = 0.0
            for v in range(self.n):
                if types[v] == mode:
                    ss += x[v] * x[v]
            norm = math.sqrt(ss)
            if norm > 0.0:
                for v in range(self.n):
                    if types[v] == mode:
                        x[v] /= norm
        return x, lam, conn

    def leading_eigen(self, weighted=False):
        """Newman's leading eigenvector communities
        (crates/engine/src/metrics/partition/leading_eigen.rs:57-160, helpers
        partition.rs:52-74, community.rs:83-146): (labels by first
        appearance, modularity on the input network, divisions). Sums run in
        the reference's order (np.cumsum is a sequential sum); eigenvectors
        come from the EISPACK restatement (symmetric_eigen)."""
        if self.directed:
            raise OracleError("The leading eigenvector method is defined here for undirected "
                              "networks only; build the network as undirected first")
        n = self.n
        if n > 3000:
            raise OracleError("the leading eigenvector method uses a dense eigendecomposition "
                              "and is limited to 3000 nodes")
        w = None
        if weighted:
            if self._w is None:
                raise OracleError("the graph has no edge weights")
            bad = np.nonzero(self._w < 0.0)[0]
            if len(bad):
                raise OracleError(f"edge {bad[0]} has negative weight {self._w[bad[0]]}; "
                                  "modularity requires non-negative weights")
            w = self._w
        src, tgt = self._src.tolist(), self._tgt.tolist()
        a = np.zeros((n, n))
        for e, (u, v) in enumerate(zip(src, tgt)):
            x = 1.0 if w is None else float(w[e])
            if u == v:
                a[u, u] += 2.0 * x
            else:
                a[u, v] += x
                a[v, u] += x
        k = np.cumsum(a, axis=1)[:, -1] if n else np.zeros(0)
        two_m = float(np.cumsum(k)[-1]) if n else 0.0
        memb = [0] * n
        splits = 0
        if two_m > 0.0:
            next_label = 1
            queue = [list(range(n))]
            while queue:
                group = queue.pop(0)
                ng = len(group)
                if ng < 2:
                    continue
                gi = np.asarray(group)
                b = a[np.ix_(gi, gi)] - np.outer(k[gi], k[gi]) / two_m
                rs = np.cumsum(b, axis=1)[:, -1]
                b[np.arange(ng), np.arange(ng)] -= rs
                scale = float(np.cumsum(np.abs(b).ravel())[-1]) / ng
                vals, vecs = symmetric_eigen(b)
                lam = float(vals[ng - 1])
                if lam != lam or lam <= 1e-10 * scale:
                    continue
                u = vecs[:, ng - 1]
                big = int(np.argmax(np.abs(u)))
                sign = -1.0 if u[big] < 0.0 else 1.0
                tiny = 1e-12 * abs(u[big])
                sv = np.where(sign * u > tiny, 1.0, -1.0)
                gain = float(np.cumsum(sv * np.cumsum(b * sv[None, :], axis=1)[:, -1])[-1])
                if gain != gain or gain <= 1e-10 * scale * ng:
                    continue
                plus = [group[r] for r in range(ng) if sv[r] > 0.0]
                minus = [group[r] for r in range(ng) if sv[r] <= 0.0]
                if not plus or not minus:
                    continue
                for v in minus:
                    memb[v] = next_label
                next_label += 1
                splits += 1
                queue.append(plus)
                queue.append(minus)
        else:
            memb = list(range(n))
        seen = {}
        labels = [seen.setdefault(c, len(seen)) for c in memb]
        kc = len(seen)
        inside, kout, kin = [0.0] * kc, [0.0] * kc, [0.0] * kc
        m = 0.0
        for e, (u, v) in enumerate(zip(src, tgt)):
            x = 1.0 if w is None else float(w[e])
            cs, ct = labels[u], labels[v]
            m += x
            kout[cs] += x
            kin[ct] += x
            if cs == ct:
                inside[cs] += x
        q = float("nan")
        if m > 0.0:
            q = 0.0
            for c in range(kc):
                kk = kout[c] + kin[c]
                q += inside[c] / m - (kk / (2.0 * m)) * (kk / (2.0 * m))
        return np.asarray(labels, dtype=np.int64), q, splits

    def centralization_eigenvector(self, normalized=True):
        """igraph's eigenvector centralization
        (crates/engine/src/metrics/topography.rs:446-498,536-548): eigenvector
        centrality with direction ignored, unweighted, loops twice, scaled
        to max 1; then n max - sum (NaN if a score is NaN), over n - 2 when
        normalized (NaN below 3 nodes); NaN for no nodes."""
        n = self.n
        if n == 0:
            return float("nan")
        x, _, _ = self.eigenvector(mode=3, weighted=False, scale=0, loops=0)
        mx = float("-inf")
        total = 0.0
        for v in x.tolist():
            mx = max(mx, v) if v == v else mx
            total += v
        if any(v != v for v in x.tolist()):
            mx = float("nan")
        raw = n * mx - total
        if not normalized:
            return raw
        return raw / (n - 2.0) if n >= 3 else float("nan")

    def katz(self, alpha=0.1, beta=1.0, mode=2, weighted=False, loops=1, normalized=True,
             tol=0.0, max_iter=0, threads=0):
        """net_katz (spectral.rs:365-407); beta is one value or n values."""
        b = np.ascontiguousarray(np.atleast_1d(beta), dtype=np.float64)
        out = np.zeros(max(self.n, 1))
        it = ctypes.c_int64()
        err = ctypes.create_string_buffer(ERR_LEN)
        if lib().orc_katz(self.h, alpha, _ptr(b), len(b), mode, int(weighted), loops,
                          int(normalized), tol, max_iter, threads, _ptr(out), ctypes.byref(it),
                          err, ERR_LEN):
            raise OracleError(err.value.decode())
        self.last_iters = it.value
        return out[: self.n]

    def bonacich(self, exponent=1.0, mode=1, weighted=False, loops=2, rescale=False, tol=0.0,
                 max_iter=0, threads=0):
        """net_bonacich_power (spectral.rs:596-655)."""
        out = np.zeros(max(self.n, 1))
        it = ctypes.c_int64()
        dense = ctypes.c_int32()
        err = ctypes.create_string_buffer(ERR_LEN)
        if lib().orc_bonacich_power(self.h, exponent, mode, int(weighted), loops, int(rescale),
                                    tol, max_iter, threads, _ptr(out), ctypes.byref(it),
                                    ctypes.byref(dense), err, ERR_LEN):
            raise OracleError(err.value.decode())
        self.last_iters = it.value
        self.last_dense = bool(dense.value)
        return out[: self.n]


    def hits(self, weighted=False, loops=0, scale=0, tol=0.0, max_iter=0, threads=0):
        """net_hits (spectral.rs:748-903): hubs, authorities, the largest
        eigenvalue of A^T A and whether the leading singular value is simple."""
        hubs = np.zeros(max(self.n, 1))
        auths = np.zeros(max(self.n, 1))
        val = ctypes.c_double()
        uniq = ctypes.c_int32()
        err = ctypes.create_string_buffer(ERR_LEN)
        if lib().orc_hits(self.h, int(weighted), loops, scale, tol, max_iter, threads,
                          _ptr(hubs), _ptr(auths), ctypes.byref(val), ctypes.byref(uniq), err,
                          ERR_LEN):
            raise OracleError(err.value.decode())
        return hubs[: self.n], auths[: self.n], val.value, bool(uniq.value)


def symmetric_eigen(a: np.ndarray):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    vals = np.zeros(n)
    vecs = np.zeros((n, n))
    if lib().orc_symmetric_eigen(n, _ptr(a), _ptr(vals), _ptr(vecs)):
        raise OracleError("symmetric eigenvalue iteration did not converge")
    return vals, vecs


def pagerank_time_op(off, cols, vals, out_strength, damping, iters, threads):
    """Seconds for `iters` reference-style PageRank iterations on a prebuilt
    pull operator (CPU baseline)."""
    n = len(off) - 1
    off = np.ascontiguousarray(off, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    vals = None if vals is None else np.ascontiguousarray(vals, dtype=np.float64)
    os_ = np.ascontiguousarray(out_strength, dtype=np.float64)
    out = np.zeros(n)
    secs = lib().orc_pagerank_time_op(n, _ptr(off), _ptr(cols), _ptr(vals), _ptr(os_), damping,
                                      iters, threads, _ptr(out))
    return secs, out


# --------------------------------------------------------------- frame graphs
# The last steps of the reference's frame builder, restated in Python loops
# for the small tables the tests use. A table is the resolved edge table:
# endpoint node indices src[e], tgt[e] over n nodes, optional weights, and
# optional missing flags (True: the row is unobserved).

NO_NODE = 0xFFFFFFFF


def _from_edges_checks(n, src, tgt, weights):
    """The checks of Graph::from_edges (crates/engine/src/graph.rs:149-192):
    the node count, every weight before any endpoint, then each edge's
    source and target in edge order. Edges are numbered as given."""
    if n > 0xFFFFFFFF:
        raise OracleError(f"node count ({n}) exceeds the supported maximum")
    if weights is not None:
        for e, x in enumerate(weights):
            if not math.isfinite(x):
                raise OracleError(f"edge {e} has a missing, NaN, or infinite weight")
    if len(src) > 0xFFFFFFFF // 2:
        raise OracleError(f"edge count ({len(src)}) exceeds the supported maximum")
    for e in range(len(src)):
        for v in (int(src[e]), int(tgt[e])):
            if v < 0 or v >= n:
                raise OracleError(
                    f"edge {e} refers to node index {v}, but valid indices are 0..{n}")


def frame_graph_of(n, src, tgt, weights=None, missing=None):
    """build_validated's observed-row pick and graph_of
    (crates/engine/src/frame/build.rs:84-88 and 106-121): the graph over all n
    nodes of the observed rows in row order. Returns (src, tgt, weights, rows)
    with rows the table row of each graph edge."""
    m = len(src)
    rows = [e for e in range(m) if missing is None or not missing[e]]
    s = [int(src[e]) for e in rows]
    t = [int(tgt[e]) for e in rows]
    w = None if weights is None else [float(weights[e]) for e in rows]
    _from_edges_checks(n, s, t, w)
    return (np.array(s, dtype=np.int64), np.array(t, dtype=np.int64),
            None if w is None else np.array(w, dtype=np.float64), np.array(rows, dtype=np.int64))


def frame_subgraph(n, src, tgt, weights, missing, keep_node, keep_edge):
    """subgraph (crates/engine/src/frame/build.rs:153-194): the nodes for which
    keep_node holds, renumbered in ascending order, and the observed rows for
    which keep_edge holds whose endpoints are both kept, in row order.
    Returns (nodes, edges, src, tgt, weights) with src/tgt renumbered."""
    index = [NO_NODE] * n
    nodes = []
    for i in range(n):
        if keep_node(i):
            index[i] = len(nodes)
            nodes.append(i)
    edges = [e for e in range(len(src))
             if (missing is None or not missing[e]) and keep_edge(e)
             and index[int(src[e])] != NO_NODE and index[int(tgt[e])] != NO_NODE]
    s = [index[int(src[e])] for e in edges]
    t = [index[int(tgt[e])] for e in edges]
    w = None if weights is None else [float(weights[e]) for e in edges]
    return (np.array(nodes, dtype=np.int64), np.array(edges, dtype=np.int64),
            np.array(s, dtype=np.int64), np.array(t, dtype=np.int64),
            None if w is None else np.array(w, dtype=np.float64))


def frame_ego_subgraph(n, src, tgt, weights, missing, node_ego, edge_ego, egos, ego):
    """ego_subgraph (crates/engine/src/frame/build.rs:220-238) on a built frame:
    the table is first checked as build does (graph_of over the observed rows).
    node_ego None: the frame has no ego role. edge_ego None: every row takes
    its source's ego (crates/engine/src/frame/validate.rs:115-117)."""
    frame_graph_of(n, src, tgt, weights, missing)
    if node_ego is None:
        raise OracleError("the frame has no ego role")
    if ego >= egos:
        raise OracleError(f"ego index {ego} is out of range; the network has {egos} ego(s)")
    if edge_ego is None:
        # unobserved rows never become edges and may hold any endpoint
        edge_ego = [node_ego[int(src[e])] if 0 <= int(src[e]) < n else -1
                    for e in range(len(src))]
    return frame_subgraph(n, src, tgt, weights, missing,
                          lambda i: node_ego[i] == ego, lambda e: edge_ego[e] == ego)


def threads_for(requested: int, items: int, work: int) -> int:
    return int(lib().orc_threads_for(requested, items, work))


if os.environ.get("KNAPPNET_ORACLE_REBUILD"):
    build(force=True)
