"""Weak and strong components on the device (net_components) against the
oracle's union-find and Tarjan's algorithm (crates/engine/src/metrics/
topography.rs:183-286): labels and counts bit-exact, on random graphs, on
shapes that stress the rounds of trimming and colouring (long paths either
way, a long cycle, chains of cycles, a cycle reached only through a long
tail), and on R-MAT graphs; eigenvector centralization (net_centralization,
topography.rs:475-498), the adjacency-matrix reading (net_graph_simplify,
topography.rs:96-141: edges, order and merged weights bit-exact) and
two-mode eigenvector centrality (net_twomode_eigenvector,
crates/engine/src/metrics/bipartite.rs:288-336) against the oracle's
restatements.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import knappnet_b200 as K
from oracle import oracle as O
from test_oracle import SplitMix64, random_case

pytestmark = pytest.mark.gpu


def check(n, src, tgt, directed):
    src = np.asarray(src, dtype=np.int64)
    tgt = np.asarray(tgt, dtype=np.int64)
    g = K.Graph(n, src, tgt, None, directed)
    og = O.Graph(n, src, tgt, None, directed)
    for strong in (False, True):
        got, cnt = g.components(strong=strong)
        ref, rcnt = og.components(strong=strong)
        assert cnt == rcnt, (strong, cnt, rcnt)
        assert np.array_equal(got.astype(np.int64), ref.astype(np.int64)), strong
    g.close()



def test_random_graphs():
    rng = SplitMix64(20241204)
    for _ in range(60):
        n, src, tgt, _, directed = random_case(rng, 40)
        check(n, src, tgt, directed)


def test_sparse_random_directed():
    rng = np.random.default_rng(7)
    for n, m in ((1000, 900), (1000, 1500), (5000, 6000), (20000, 40000)):
        check(n, rng.integers(0, n, m), rng.integers(0, n, m), True)


def test_paths_and_cycles():
    L = 3000
    a = np.arange(L - 1)
    check(L, a, a + 1, True)            # forward path: L trivial components
    check(L, a + 1, a, True)            # backward path
    c = np.arange(L)
    check(L, c, (c + 1) % L, True)      # one cycle
    # cycles of 5 chained by one arc each, in both id orders
    k = 400
    s, t = [], []
    for b in range(k):
        base = 5 * b
        for i in range(5):
            s.append(base + i)
            t.append(base + (i + 1) % 5)
        if b + 1 < k:
            s.append(base)
            t.append(base + 5)
    check(5 * k, s, t, True)
    check(5 * k, t, s, True)
    # a long tail into a cycle, loops and parallel arcs on the way
    tail = 2000
    s = list(range(tail)) + [tail, tail + 1, tail + 2, 5, 5]
    t = list(range(1, tail + 1)) + [tail + 1, tail + 2, tail, 5, 6]
    check(tail + 3, s, t, True)


def test_empty_and_isolated():
    check(1, [], [], True)
    check(7, [], [], True)
    check(4, [0, 1], [0, 1], True)


@pytest.mark.parametrize("scale", [14, 18])
def test_rmat_directed(scale):
    g = K.generate_rmat(scale, 16, seed=20241205 + scale, clean=True)
    s, t, _ = g.edges()
    n = g.n
    g.close()
    check(n, s, t, True)


def test_eigenvector_centralization_matches_oracle():
    rng = SplitMix64(20241206)
    for _ in range(20):
        n, src, tgt, _, directed = random_case(rng, 30)
        src = np.asarray(src, dtype=np.int64)
        tgt = np.asarray(tgt, dtype=np.int64)
        g = K.Graph(n, src, tgt, None, directed)
        og = O.Graph(n, src, tgt, None, directed)
        try:
            ref = og.centralization_eigenvector()
        except RuntimeError:
            with pytest.raises(RuntimeError):
                g.centralization_eigenvector()
            continue
        got = g.centralization_eigenvector()
        if np.isnan(ref):
            assert np.isnan(got)
        else:
            assert abs(got - ref) <= 1e-9 + 1e-8 * abs(ref), (got, ref)
        raw = g.centralization(normalized=False)
        assert abs(raw - og.centralization_eigenvector(normalized=False)) <= 1e-9 * max(1, n)
        g.close()



def test_centralization_codes():
    g = K.Graph(4, np.array([0, 1, 2]), np.array([1, 2, 3]), None, True)
    for kw, msg in (({"measure": 4}, "unknown centralization measure code 4"),
                    ({"mode": 0}, "unknown degree mode code 0"),
                    ({"convention": 5}, "unknown convention code 5"),
                    ({"convention": 1}, "NetworkX has no centralization index"),
                    ({"convention": 2}, "igraph convention only, not sna"),
                    ({"mode": 1}, "direction ignored"),
                    ({"measure": 0}, "outside this library")):
        with pytest.raises(RuntimeError, match=msg):
            g.centralization(**kw)
    memb = np.zeros(4, dtype=np.int32)
    cnt = ctypes.c_int64()
    err = ctypes.create_string_buffer(256)
    assert K.lib().net_components(g.h, 2, memb.ctypes.data, ctypes.byref(cnt), err, 256) == 1
    assert err.value.decode() == "unknown component kind code 2"
    g.close()


def test_simplify_matches_oracle():
    """net_graph_simplify vs the oracle's restatement of simplify
    (topography.rs:96-141): the same edges in the same order and the same
    merged weights, bit-exact."""
    rng = SplitMix64(20241207)
    for case in range(40):
        n, src, tgt, w, directed = random_case(rng, 30)
        weights = np.asarray(w) if case % 2 else None
        g = K.Graph(n, np.asarray(src), np.asarray(tgt), weights, directed)
        og = O.Graph(n, np.asarray(src), np.asarray(tgt), weights, directed)
        for undirected in (False, True):
            for keep in (0, 1):
                a = g.simplify(undirected=undirected, keep=keep)
                b = og.simplify(undirected=undirected, keep=keep)
                sa, ta, wa = a.edges()
                sb, tb, wb = b.edges()
                assert a.directed == b.directed
                assert np.array_equal(sa, sb) and np.array_equal(ta, tb), (case, undirected, keep)
                if weights is None:
                    assert wa is None
                else:
                    assert np.array_equal(wa, wb), (case, undirected, keep)
                a.close()
        g.close()
    # a heavy multigraph: 200,000 arcs over 300 nodes
    r = np.random.default_rng(11)
    s, t = r.integers(0, 300, 200_000), r.integers(0, 300, 200_000)
    w = r.uniform(0.1, 5.0, 200_000)
    g = K.Graph(300, s, t, w, True)
    og = O.Graph(300, s, t, w, True)
    for undirected, keep in ((False, 0), (True, 1)):
        sa, ta, wa = g.simplify(undirected, keep).edges()
        sb, tb, wb = og.simplify(undirected, keep).edges()
        assert np.array_equal(sa, sb) and np.array_equal(ta, tb) and np.array_equal(wa, wb)
    with pytest.raises(RuntimeError, match="unknown parallel-edge weight code 2"):
        g.simplify(keep=2)
    g.close()


def bipartite_case(r, n1, n2, m):
    s = r.integers(0, n1, m)
    t = n1 + r.integers(0, n2, m)
    flip = r.random(m) < 0.5
    src, tgt = np.where(flip, t, s), np.where(flip, s, t)
    return n1 + n2, src, tgt, [0] * n1 + [1] * n2


def test_twomode_eigenvector_matches_oracle():
    r = np.random.default_rng(12)
    for n1, n2, m, directed in ((5, 7, 12, False), (20, 30, 90, True), (50, 8, 400, False),
                                (300, 200, 3000, True), (40, 40, 0, False)):
        n, src, tgt, types = bipartite_case(r, n1, n2, m)
        g = K.Graph(n, src, tgt, None, directed)
        og = O.Graph(n, src, tgt, None, directed)
        x, lam, conn = g.twomode_eigenvector(types)
        rx, rlam, rconn = og.twomode_eigenvector(types)
        assert conn == rconn
        if m == 0:
            assert np.isnan(x).all() and lam == 0.0
        else:
            assert abs(lam - rlam) <= 1e-10 * rlam
            assert np.nanmax(np.abs(x - rx)) <= 1e-9, (n1, n2, m)
            for mode in (0, 1):
                sel = np.asarray(types) == mode
                assert abs(np.sum(x[sel] ** 2) - 1.0) <= 1e-12
        g.close()


def test_twomode_eigenvector_errors():
    g = K.Graph(4, np.array([0, 1, 0]), np.array([2, 3, 1]), None, False)
    with pytest.raises(RuntimeError, match="node 1 has type code 2; use 0 for the first mode"):
        g.twomode_eigenvector([0, 2, 1, 1])
    with pytest.raises(RuntimeError, match="edge 2 joins nodes 0 and 1, which are in the same mode"):
        g.twomode_eigenvector([0, 0, 1, 1])
    g.close()


def planted(r, sizes, p_in, p_out, weighted=False, isolates=0):
    """Undirected planted-partition multigraph: blocks of the given sizes,
    then `isolates` nodes without ties."""
    n = sum(sizes) + isolates
    block = np.repeat(np.arange(len(sizes)), sizes)
    s, t = [], []
    nb = sum(sizes)
    for u in range(nb):
        for v in range(u + 1, nb):
            if r.random() < (p_in if block[u] == block[v] else p_out):
                s.append(u)
                t.append(v)
    w = r.uniform(0.5, 2.0, len(s)) if weighted else None
    return n, np.asarray(s, dtype=np.int64), np.asarray(t, dtype=np.int64), w


@pytest.mark.parametrize("case", range(6))
def test_leading_eigen_matches_oracle(case):
    """net_leading_eigen vs the oracle (EISPACK eigenvectors, the reference's
    summation order): the same labels, the same number of divisions, the
    modularity within 1e-12 relative."""
    r = np.random.default_rng(100 + case)
    shapes = [([30, 30, 30], 0.3, 0.02, False, 0), ([50, 40, 30, 20], 0.25, 0.01, True, 5),
              ([120], 0.05, 0.0, False, 0), ([60, 60], 0.2, 0.05, True, 3),
              ([200, 150, 100, 50], 0.08, 0.004, False, 10), ([25] * 12, 0.5, 0.01, True, 0)]
    sizes, p_in, p_out, weighted, iso = shapes[case]
    n, s, t, w = planted(r, sizes, p_in, p_out, weighted, iso)
    g = K.Graph(n, s, t, w, False)
    og = O.Graph(n, s, t, w, False)
    memb, q, splits = g.leading_eigen(weighted=weighted)
    rm, rq, rsplits = og.leading_eigen(weighted=weighted)
    assert splits == rsplits
    assert np.array_equal(memb, rm)
    assert abs(q - rq) <= 1e-12 * abs(rq) + 1e-14
    g.close()


def test_leading_eigen_reference_cases_and_errors():
    """The reference's own cases (partition/leading_eigen.rs:163-206)."""
    g = K.Graph(6, np.array([0, 0, 1, 3, 3, 4, 2]), np.array([1, 2, 2, 4, 5, 5, 3]), None, False)
    memb, q, splits = g.leading_eigen()
    assert memb.tolist() == [0, 0, 0, 1, 1, 1] and splits == 1
    assert abs(q - 5.0 / 14.0) < 1e-14
    s, t = [], []
    for c in range(4):
        for i in range(5):
            for j in range(i + 1, 5):
                s.append(5 * c + i)
                t.append(5 * c + j)
        s.append(5 * c)
        t.append((5 * c + 5) % 20)
    memb, _, splits = K.Graph(20, np.array(s), np.array(t), None, False).leading_eigen()
    assert splits == 3
    for c in range(4):
        assert len(set(memb[5 * c: 5 * c + 5].tolist())) == 1
    s, t = zip(*[(i, j) for i in range(5) for j in range(i + 1, 5)])
    memb, _, splits = K.Graph(5, np.array(s), np.array(t), None, False).leading_eigen()
    assert memb.tolist() == [0] * 5 and splits == 0
    memb, q, _ = K.Graph(3, np.array([], dtype=np.int64), np.array([], dtype=np.int64), None,
                         False).leading_eigen()
    assert memb.tolist() == [0, 1, 2] and np.isnan(q)
    with pytest.raises(RuntimeError, match="undirected networks only"):
        K.Graph(2, np.array([0]), np.array([1]), None, True).leading_eigen()
    with pytest.raises(RuntimeError, match="the graph has no edge weights"):
        K.Graph(2, np.array([0]), np.array([1]), None, False).leading_eigen(weighted=True)
    with pytest.raises(RuntimeError, match="limited to 3000 nodes"):
        K.Graph(3001, np.array([0]), np.array([1]), None, False).leading_eigen()


def test_zero_node_graph_every_entry_point():
    """A graph without nodes: every entry point gives what the oracle gives
    (equal results, NaN where undefined), or both refuse."""
    e = np.array([], dtype=np.int64)
    for directed in (True, False):
        g = K.Graph(0, e, e, None, directed)
        og = O.Graph(0, e, e, None, directed)
        calls = [
            ("components", lambda x: x.components(strong=True)[1]),
            ("weak", lambda x: x.components(strong=False)[1]),
            ("pagerank", lambda x: x.pagerank()),
            ("eigenvector", lambda x: x.eigenvector(mode=3)[0]),
            ("katz", lambda x: x.katz(alpha=0.1)),
            ("hits", lambda x: x.hits()[0]),
            ("centralization", lambda x: x.centralization_eigenvector()),
            ("twomode", lambda x: x.twomode_eigenvector([])[0]),
        ]
        if not directed:
            calls.append(("leading_eigen", lambda x: x.leading_eigen()[0]))
        for name, fn in calls:
            try:
                ref = fn(og)
            except RuntimeError:
                with pytest.raises(RuntimeError):
                    fn(g)
                continue
            got = fn(g)
            assert np.array_equal(np.asarray(got, dtype=np.float64),
                                  np.asarray(ref, dtype=np.float64), equal_nan=True), name
        sg = g.simplify(undirected=True)
        assert sg.n == 0 and sg.m == 0
        sg.close()
        g.close()
