"""Pins the CPU oracle against the reference's own golden files and
known-answer tests, before anything is checked against it.

Sources of the expected values:
- validation/golden/{definition,networkx}/<fixture>/<variant>.csv, packed in
  tests/golden/spectral_golden.json by tests/golden/make_golden.py;
- the reference's unit tests: Philox KATs (crates/engine/src/rng.rs:116-134),
  CSR layout (graph.rs:354-372), degree (metrics/degree.rs:79-98), PageRank
  hand values (metrics/spectral.rs:953-989), eigenvector closed forms
  (metrics/eigenvector.rs:1151-1254);
- the reference's property tests (crates/engine/tests/spectral_properties.rs).
"""
from __future__ import annotations

import math

import numpy as np
import pytest

import goldens
from oracle import oracle as O


# ------------------------------------------------------------------ golden files
@pytest.mark.parametrize("fx_name,variant,orc", goldens.cases())
def test_oracle_matches_golden(fx_name, variant, orc):
    doc = goldens.load()
    fx = doc["fixtures"][fx_name]
    g = goldens.make_graph(O.Graph, fx)
    got = goldens.run_variant(g, fx, variant)
    ok, msg = goldens.agree_variant(got, doc["golden"][fx_name][variant][orc], variant)
    assert ok, msg


def test_golden_coverage():
    # Every PageRank and eigenvector variant is pinned on most fixtures.
    per_variant = {}
    for _, variant, _ in goldens.cases():
        per_variant[variant] = per_variant.get(variant, 0) + 1
    assert per_variant["pagerank"] >= 28
    assert per_variant["eigenvector"] >= 27
    assert per_variant["pagerank_weighted"] >= 7


# ------------------------------------------------------------------ Philox
def test_philox_known_answers():
    # Random123 known-answer vectors (rng.rs:116-134).
    assert list(O.philox([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    m = 0xFFFFFFFF
    assert list(O.philox([m] * 4, [m, m])) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert list(O.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344],
                         [0xA4093822, 0x299F31D0])) == [0xD16CFE09, 0x94FDCCEB, 0x5001E420,
                                                        0x24126EA1]


def test_streams_reproducible_and_distinct():
    a = O.stream_u32(7, 3, 8)
    assert (a == O.stream_u32(7, 3, 8)).all()
    assert not (a == O.stream_u32(7, 4, 8)).all()
    assert not (a == O.stream_u32(8, 3, 8)).all()
    # Stream words are the Philox blocks of counter (block, stream) in order.
    blk0 = O.philox([0, 0, 3, 0], [7, 0])
    blk1 = O.philox([1, 0, 3, 0], [7, 0])
    assert list(a) == list(blk0) + list(blk1)
    b = O.stream_below(7, 3, 10, 1000)
    assert b.max() < 10 and len(set(b.tolist())) == 10


# ------------------------------------------------------------------ graph build
def test_csr_layout_directed():
    # graph.rs:354-362.
    g = O.Graph(4, [2, 0, 0, 1, 0], [1, 3, 1, 2, 1], None, True)
    off, tgt, _ = g.csr(0)
    rows = [tgt[off[v]:off[v + 1]].tolist() for v in range(4)]
    assert rows[0] == [1, 1, 3] and rows[1] == [2] and rows[2] == [1]
    off, tgt, _ = g.csr(1)
    assert tgt[off[1]:off[2]].tolist() == [0, 0, 2]
    assert tgt[off[3]:off[4]].tolist() == [0]


def test_csr_layout_undirected():
    # graph.rs:364-372.
    g = O.Graph(3, [0, 1, 2], [1, 2, 2], [1.0, 2.0, 3.0], False)
    off, tgt, w = g.csr(0)
    assert tgt[off[1]:off[2]].tolist() == [0, 2]
    assert w[off[1]:off[2]].tolist() == [1.0, 2.0]
    assert tgt[off[2]:off[3]].tolist() == [1, 2]
    assert w[off[2]:off[3]].tolist() == [2.0, 3.0]


def test_parallel_arcs_keep_input_order():
    g = O.Graph(3, [0, 0, 0, 1], [2, 1, 2, 0], [5.0, 6.0, 7.0, 8.0], True)
    off, tgt, w = g.csr(0)
    assert tgt[off[0]:off[1]].tolist() == [1, 2, 2]
    assert w[off[0]:off[1]].tolist() == [6.0, 5.0, 7.0]


def test_rejects_bad_input():
    with pytest.raises(O.OracleError, match="refers to node index 2"):
        O.Graph(2, [0], [2], None, True)
    with pytest.raises(O.OracleError, match="NaN"):
        O.Graph(2, [0], [1], [float("nan")], True)


def test_degree_known_answers():
    # metrics/degree.rs:79-98.
    g = O.Graph(3, [0, 0, 1, 2], [1, 1, 1, 0], None, True)
    assert g.degree(1, True).tolist() == [2, 1, 1]
    assert g.degree(2, True).tolist() == [1, 3, 0]
    assert g.degree(3, True).tolist() == [3, 4, 1]
    assert g.degree(3, False).tolist() == [3, 2, 1]
    u = O.Graph(3, [0, 0, 1, 2], [1, 1, 1, 0], None, False)
    assert u.degree(3, True).tolist() == [3, 4, 1]


# ------------------------------------------------------------------ PageRank
def small():
    # 0 -> 1, 0 -> 2, 1 -> 2, 2 -> 0, 3 -> 2, 2 -> 4 (spectral.rs:948-951).
    return O.Graph(5, [0, 0, 1, 2, 3, 2], [1, 2, 2, 0, 2, 4], None, True)


def test_pagerank_hand_values():
    # spectral.rs:953-989.
    g = small()
    want = [0.2142011097, 0.1574496602, 0.3477339318, 0.0664141886, 0.2142011097]
    assert np.allclose(g.pagerank(), want, atol=1e-9, rtol=0)
    p = [1.0, 0.0, 0.0, 0.0, 0.0]
    want = [0.3928645968, 0.1669674536, 0.3088897892, 0.0, 0.1312781604]
    assert np.allclose(g.pagerank(personalization=p), want, atol=1e-9, rtol=0)
    want = [0.3166510816, 0.1629073936, 0.3254597594, 0.0283306839, 0.1666510816]
    assert np.allclose(g.pagerank(personalization=p, dangling=1), want, atol=1e-9, rtol=0)
    with pytest.raises(O.OracleError, match="damping"):
        g.pagerank(damping=1.5)


class SplitMix64:
    """spectral_properties.rs:21-37."""

    def __init__(self, seed):
        self.s = seed & (2**64 - 1)

    def next(self):
        M = 2**64 - 1
        self.s = (self.s + 0x9E3779B97F4A7C15) & M
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    def below(self, n):
        return self.next() % n

    def unit(self):
        return (self.next() >> 11) / float(1 << 53)


def random_case(rng, max_n):
    """spectral_properties.rs:47-64."""
    n = 2 + rng.below(max_n)
    m = rng.below(n * n // 3 + 2)
    directed = rng.below(2) == 0
    src, tgt, w = [], [], []
    for _ in range(m):
        src.append(rng.below(n))
        tgt.append(rng.below(n))
        w.append(0.25 + 3.0 * rng.unit())
    return n, src, tgt, w, directed


def dense(n, src, tgt, w, directed, weighted, into, loop_factor):
    """spectral_properties.rs:88-115."""
    a = np.zeros((n, n))
    for k, (s, t) in enumerate(zip(src, tgt)):
        x = w[k] if weighted else 1.0
        if s == t:
            f = min(loop_factor, 1.0) if directed else loop_factor
            a[s, s] += f * x
        elif directed:
            if into:
                a[t, s] += x
            else:
                a[s, t] += x
        else:
            a[s, t] += x
            a[t, s] += x
    return a


def test_pagerank_is_stationary_and_relabel_invariant():
    # spectral_properties.rs:190-222.
    rng = SplitMix64(21)
    for _ in range(150):
        n, src, tgt, w, directed = random_case(rng, 30)
        weighted = rng.below(2) == 0
        g = O.Graph(n, src, tgt, w if weighted else None, directed)
        x = g.pagerank(weighted=weighted, threads=1)
        assert abs(x.sum() - 1.0) < 1e-12
        a = dense(n, src, tgt, w, directed, weighted, False, 2.0)
        out = a.sum(axis=1)
        stuck = x[out == 0].sum()
        for i in range(n):
            flow = sum(a[j, i] / out[j] * x[j] for j in range(n) if out[j] > 0)
            rhs = 0.85 * (flow + stuck / n) + 0.15 / n
            assert abs(x[i] - rhs) < 1e-10
        perm = list(range(n))
        for i in range(n - 1, 0, -1):
            j = rng.below(i + 1)
            perm[i], perm[j] = perm[j], perm[i]
        h = O.Graph(n, [perm[v] for v in src], [perm[v] for v in tgt],
                    w if weighted else None, directed)
        y = h.pagerank(weighted=weighted, threads=1)
        back = np.array([y[perm[v]] for v in range(n)])
        assert np.all(np.abs(x - back) <= 1e-9 * (1 + np.maximum(np.abs(x), np.abs(back))))


# ------------------------------------------------------------------ eigenvector
def test_star_closed_form():
    g = O.Graph(5, [0, 0, 0, 0], [1, 2, 3, 4], None, False)
    v, lam, conn = g.eigenvector()
    assert abs(lam - 2.0) < 1e-10 and conn
    assert np.allclose(v, [1.0, 0.5, 0.5, 0.5, 0.5], atol=1e-10, rtol=0)
    u, _, _ = g.eigenvector(scale=1)
    assert abs((u * u).sum() - 1.0) < 1e-12


def test_path_golden_ratio():
    g = O.Graph(4, [0, 1, 2], [1, 2, 3], None, False)
    v, lam, _ = g.eigenvector()
    phi = (1 + 5 ** 0.5) / 2
    assert abs(lam - phi) < 1e-10
    assert np.allclose(v, [1 / phi, 1, 1, 1 / phi], atol=1e-10, rtol=0)


def test_directed_modes():
    g = O.Graph(3, [0, 1, 2, 2], [1, 2, 0, 1], None, True)
    ins, li, _ = g.eigenvector(mode=2)
    outs, lo, _ = g.eigenvector(mode=1)
    a = np.array([[0.0, 1, 0], [0, 0, 1], [1, 1, 0]])
    assert np.allclose(a.T @ ins, li * ins, atol=1e-10)
    assert np.allclose(a @ outs, lo * outs, atol=1e-10)
    assert ins[1] > ins[0]


def test_loops_and_weights():
    g = O.Graph(2, [0, 0], [0, 1], [1.0, 3.0], False)
    _, lam, _ = g.eigenvector()
    assert abs(lam - (1 + 2 ** 0.5)) < 1e-10
    _, lam, _ = g.eigenvector(loops=1, weighted=True)
    assert abs(lam - (1 + 37 ** 0.5) / 2) < 1e-10
    neg = O.Graph(2, [0], [1], [-1.0], False)
    with pytest.raises(O.OracleError, match="negative"):
        neg.eigenvector(weighted=True)


def test_acyclic_and_empty():
    e = O.Graph(3, [], [], None, False)
    v, lam, conn = e.eigenvector()
    assert v.tolist() == [1.0, 1.0, 1.0] and lam == 0.0 and not conn
    dag = O.Graph(3, [0, 1], [1, 2], None, True)
    assert dag.eigenvector(mode=2)[0].tolist() == [0.0, 0.0, 1.0]
    assert dag.eigenvector(mode=1)[0].tolist() == [1.0, 0.0, 0.0]


def test_disconnected_flagged():
    g = O.Graph(5, [0, 1, 2, 3], [1, 2, 0, 4], None, False)
    v, lam, conn = g.eigenvector()
    assert not conn and abs(lam - 2.0) < 1e-10
    assert np.allclose(v, [1, 1, 1, 0, 0], atol=1e-9, rtol=0)


def test_lanczos_eigen_equation_and_relabel():
    # spectral_properties.rs:129-160 (fewer cases; the property is the same).
    rng = SplitMix64(11)
    for _ in range(80):
        n, src, tgt, w, _ = random_case(rng, 40)
        weighted = rng.below(2) == 0
        g = O.Graph(n, src, tgt, w if weighted else None, False)
        x, lam, _ = g.eigenvector(weighted=weighted, scale=1, threads=1)
        if lam == 0.0:
            continue
        a = dense(n, src, tgt, w, False, weighted, True, 2.0)
        y = a @ x
        assert (x >= 0).all()
        assert np.all(np.abs(y - lam * x) <= 1e-9 * (1 + lam))


def test_thread_count_does_not_change_results():
    # eigenvector.rs:1256-1283 and spectral_properties.rs:162-188.
    n = 3000
    s, t = [], []
    for i in range(n):
        for d in (1, 7, 31, 101, 997, 1999):
            s.append(i)
            t.append((i * d + 3) % n)
    g = O.Graph(n, s, t, None, True)
    a = g.eigenvector(threads=1)
    b = g.eigenvector(threads=4)
    assert (a[0] == b[0]).all() and a[1] == b[1]
    pa = g.pagerank(threads=1)
    pb = g.pagerank(threads=4)
    assert (pa == pb).all()


def test_symmetric_eigen_matches_numpy():
    rng = np.random.default_rng(3)
    for n in (1, 2, 5, 12, 20):
        a = rng.standard_normal((n, n))
        a = a + a.T
        vals, vecs = O.symmetric_eigen(a)
        assert np.allclose(vals, np.linalg.eigvalsh(a), atol=1e-12)
        assert np.allclose(a @ vecs, vecs * vals, atol=1e-10)
        assert (np.diff(vals) >= 0).all()


# ------------------------------------------------------------------ generators
def test_gnm_is_simple_and_sorted():
    f, t = O.gnm(10_000, 50_000, directed=False, seed=1)
    assert len(f) == 50_000
    assert (f < t).all()
    key = f.astype(np.uint64) << np.uint64(32) | t.astype(np.uint64)
    assert (np.diff(key.astype(np.int64)) > 0).all()
    f2, t2 = O.gnm(10_000, 50_000, directed=False, seed=1)
    assert (f == f2).all() and (t == t2).all()


def test_rmat_quadrant_frequencies():
    s, t = O.rmat_raw(1, 200_000, 0.57, 0.19, 0.19, seed=5)
    q = s * 2 + t
    freq = np.bincount(q, minlength=4) / len(q)
    assert np.allclose(freq, [0.57, 0.19, 0.19, 0.05], atol=0.01)


def test_rmat_cleaning_and_lognormal_strengths():
    """The generators the benchmark's reference arm uses: cleaned R-MAT edges
    (self-loops and duplicates removed, sorted by (source, target); or each
    unordered pair once) and lognormal strengths from Box-Muller on the
    edge's Philox stream, computed here one value at a time."""
    scale = 11
    r, q = O.rmat_raw(scale, 16 << scale, 0.57, 0.19, 0.19, seed=77)
    keep = r != q
    key = np.unique(r[keep].astype(np.int64) << scale | q[keep].astype(np.int64))
    s, t = O.rmat(scale, 16, 0.57, 0.19, 0.19, 77)
    assert np.array_equal(s, key >> scale) and np.array_equal(t, key & ((1 << scale) - 1))
    lo = np.minimum(r, q)[keep].astype(np.int64)
    hi = np.maximum(r, q)[keep].astype(np.int64)
    key = np.unique(lo << scale | hi)
    s, t = O.rmat(scale, 16, 0.57, 0.19, 0.19, 77, symmetrize=True)
    assert np.array_equal(s, key >> scale) and np.array_equal(t, key & ((1 << scale) - 1))
    raw = O.rmat(scale, 16, 0.57, 0.19, 0.19, 77, clean=False)
    assert np.array_equal(raw[0], r) and np.array_equal(raw[1], q)
    w = O.lognormal(500, 5)
    u = np.array([O.stream_u32(5, e, 4) for e in range(500)], dtype=np.uint64)
    a = (u[:, 0] << np.uint64(32) | u[:, 1]) >> np.uint64(11)
    b = (u[:, 2] << np.uint64(32) | u[:, 3]) >> np.uint64(11)
    z = (np.sqrt(-2 * np.log(1 - a.astype(np.float64) / 2.0 ** 53))
         * np.cos(2 * np.pi * (b.astype(np.float64) / 2.0 ** 53)))
    want = np.exp(z).astype(np.float32).astype(np.float64)
    assert np.abs(w / want - 1).max() <= 2 ** -23


# ------------------------------------------------------------------ Katz, Bonacich
def katz_bonacich_known_answers(G, err):
    """The reference's hand values (crates/engine/src/metrics/spectral.rs:
    992-1040), on an engine whose graphs are built by G(n, src, tgt, w,
    directed) and whose failures raise `err`."""
    # 0 -> 1 -> 2: x = 1 + alpha A^T x gives 1, 1 + a, 1 + a + a^2
    dag = G(3, [0, 1], [1, 2], None, True)
    assert np.array_equal(dag.katz(alpha=10.0, normalized=False), [1.0, 11.0, 111.0])
    small = G(5, [0, 0, 1, 2, 3, 2], [1, 2, 2, 0, 2, 4], None, True)
    want = [1.3445378151, 1.2689075630, 1.7226890756, 1.0, 1.3445378151]
    assert np.allclose(small.katz(alpha=0.2, normalized=False, loops=2), want, atol=1e-9, rtol=0)
    with pytest.raises(err, match="lambda_max"):
        small.katz(alpha=0.76, normalized=False, loops=2)
    # star around 0 with an extra edge 1 - 4
    star = G(5, [0, 0, 0, 1], [1, 2, 3, 4], None, False)
    assert np.allclose(star.bonacich(exponent=0.5),
                       [1.4696735043, 1.1238679739, 0.7780624435, 0.7780624435, 0.6051596782],
                       atol=1e-9, rtol=0)
    assert np.allclose(star.bonacich(exponent=-0.5),
                       [1.8605210188, -0.6201736729, -0.6201736729, -0.6201736729,
                        0.6201736729], atol=1e-9, rtol=0)
    assert abs(star.bonacich(exponent=0.5, rescale=True).sum() - 1.0) < 1e-12
    # exponent 1 lies beyond 1 / lambda_max (about 1.9): the dense solve,
    # (I - A) y proportional to A 1, squares summing to n
    y = star.bonacich(exponent=1.0)
    a = np.zeros((5, 5))
    for s, t in ((0, 1), (0, 2), (0, 3), (1, 4)):
        a[s, t] = a[t, s] = 1.0
    lhs, rhs = (np.eye(5) - a) @ y, a @ np.ones(5)
    k = lhs @ rhs / (rhs @ rhs)
    assert np.allclose(lhs, k * rhs, atol=1e-9)
    assert abs((y * y).sum() - 5.0) < 1e-9
    # errors the reference raises
    with pytest.raises(err, match="alpha"):
        small.katz(alpha=-1.0)
    with pytest.raises(err):
        small.katz(alpha=0.1, beta=[1.0, 2.0])
    with pytest.raises(err, match="finite"):
        star.bonacich(exponent=float("inf"))


def test_oracle_katz_bonacich_known_answers():
    katz_bonacich_known_answers(O.Graph, O.OracleError)
    g = O.Graph(5, [0, 0, 0, 1], [1, 2, 3, 4], None, False)
    g.bonacich(exponent=1.0)
    assert g.last_dense
    g.bonacich(exponent=0.5)
    assert not g.last_dense


# ------------------------------------------------------------------ HITS
def hits_known_answers(G):
    """The reference's hand values (spectral.rs:1073-1092)."""
    small = G(5, [0, 0, 1, 2, 3, 2], [1, 2, 2, 0, 2, 4], None, True)
    hubs, auths, value, unique = small.hits()
    h = 0.5 ** 0.5
    assert np.allclose(hubs, [1.0, h, 0.0, h, 0.0], atol=1e-9, rtol=0)
    assert np.allclose(auths, [0.0, 2 ** 0.5 - 1.0, 1.0, 0.0, 0.0], atol=1e-9, rtol=0)
    assert unique
    # a directed 4-cycle: A^T A = I, every block ties, equal scores stay put
    cyc = G(4, [0, 1, 2, 3], [1, 2, 3, 0], None, True)
    hubs, _, _, unique = cyc.hits()
    assert not unique
    assert np.array_equal(hubs, [1.0] * 4)
    empty = G(3, [], [], None, True)
    hubs, auths, value, _ = empty.hits()
    assert np.isnan(hubs).all() and np.isnan(auths).all() and value == 0.0


def test_oracle_hits_known_answers():
    hits_known_answers(O.Graph)
