"""Parity of the device frame-graph builder (net_frame_graph, net_frame_egos)
with the oracle's restatement of the reference's graph_of, subgraph and
ego_subgraph (crates/engine/src/frame/build.rs:84-121, 153-194, 220-238).

Bars: graph structure, edge order, table rows and node mappings bit-exact;
per-ego PageRank of the packed ego graph within 1e-12 L1 of the oracle's
PageRank of each ego subgraph built on its own, with the same iteration
counts; error messages as Graph::from_edges words them."""
from __future__ import annotations

import numpy as np
import pytest

import knappnet_b200 as K
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def random_table(seed, n, m, egos, weighted=True, miss_frac=0.1, bad_missing=True):
    """A resolved edge table whose unobserved rows may hold anything (bad
    endpoints, non-finite weights): they must never be read as edges."""
    rng = np.random.default_rng(seed)
    node_ego = rng.integers(-1, egos, size=n) if egos else np.full(n, -1)
    # most rows stay inside one ego so that ego graphs have edges
    src = rng.integers(0, n, size=m)
    tgt = rng.integers(0, n, size=m)
    for e in range(m):
        k = node_ego[src[e]]
        if k >= 0 and rng.random() < 0.8:
            members = np.flatnonzero(node_ego == k)
            tgt[e] = members[rng.integers(0, len(members))]
    edge_ego = np.where(rng.random(m) < 0.9, node_ego[src], rng.integers(-1, max(egos, 1), m))
    w = rng.lognormal(size=m) if weighted else None
    missing = rng.random(m) < miss_frac
    if bad_missing and missing.any():
        idx = np.flatnonzero(missing)
        src[idx[::3]] = n + 5
        tgt[idx[1::3]] = -2
        if w is not None:
            w[idx[2::3]] = np.nan
    return src, tgt, w, missing, node_ego, edge_ego


def oracle_packed_egos(n, src, tgt, w, missing, node_ego, edge_ego, egos):
    parts = [O.frame_ego_subgraph(n, src, tgt, w, missing, node_ego, edge_ego, egos, k)
             for k in range(egos)]
    off = np.concatenate([[0], np.cumsum([len(p[0]) for p in parts])]).astype(np.int64)
    return parts, off


@pytest.mark.parametrize("directed,weighted", [(True, True), (False, False), (True, False)])
def test_frame_graph_matches_graph_of(directed, weighted):
    n, m = 700, 5000
    src, tgt, w, missing, _, _ = random_table(3, n, m, 0, weighted)
    g, rows = K.frame_graph(n, src, tgt, w, missing, directed)
    s, t, ww, orows = O.frame_graph_of(n, src, tgt, w, missing)
    gs, gt, gw = g.edges()
    assert g.n == n and g.m == len(orows)
    assert np.array_equal(rows, orows)
    assert np.array_equal(gs, s) and np.array_equal(gt, t)
    if weighted:
        assert np.array_equal(gw, ww)
    # the CSR the library built from it is the oracle graph's CSR
    og = O.Graph(n, s, t, ww, directed)
    for which in ((0, 1) if directed else (0,)):
        off, cols, cw = g.csr(which)[:3]
        ooff, ocols, ocw = og.csr(which)
        assert np.array_equal(off.astype(np.uint64), ooff) and np.array_equal(cols, ocols)
        if weighted:
            assert np.array_equal(cw, ocw)
    ref = og.pagerank(weighted=weighted, directed=directed, tol=1e-12)
    got = g.pagerank(weighted=weighted, directed=directed, tol=1e-12)
    assert np.abs(got - ref).sum() <= 1e-12


def test_frame_graph_without_flags_and_empty_tables():
    src, tgt = np.array([0, 1, 2, 2]), np.array([1, 2, 0, 0])
    g, rows = K.frame_graph(3, src, tgt)
    assert rows.tolist() == [0, 1, 2, 3] and g.m == 4
    g, rows = K.frame_graph(3, src, tgt, missing=np.ones(4, dtype=bool))
    assert g.m == 0 and g.n == 3 and len(rows) == 0
    assert np.allclose(g.pagerank(), 1 / 3)
    g, rows = K.frame_graph(5, np.array([], dtype=np.int64), np.array([], dtype=np.int64))
    assert g.m == 0 and g.n == 5
    g, rows = K.frame_graph(0, np.array([], dtype=np.int64), np.array([], dtype=np.int64))
    assert g.m == 0 and g.n == 0


@pytest.mark.parametrize("edge_labels", [True, False])
@pytest.mark.parametrize("directed,weighted", [(True, True), (False, True), (True, False)])
def test_frame_egos_match_ego_subgraph(directed, weighted, edge_labels):
    n, m, egos = 600, 4000, 9
    src, tgt, w, missing, node_ego, edge_ego = random_table(11, n, m, egos, weighted)
    if not edge_labels:
        edge_ego = None
    g, off, ids, rows = K.frame_egos(n, src, tgt, node_ego, edge_ego, egos, w, missing, directed)
    parts, ooff = oracle_packed_egos(n, src, tgt, w, missing, node_ego, edge_ego, egos)
    assert np.array_equal(off, ooff)
    assert np.array_equal(ids, np.concatenate([p[0] for p in parts]))
    assert np.array_equal(rows, np.concatenate([p[1] for p in parts]))
    gs, gt, gw = g.edges()
    assert np.array_equal(gs, np.concatenate([p[2] + ooff[k] for k, p in enumerate(parts)]))
    assert np.array_equal(gt, np.concatenate([p[3] + ooff[k] for k, p in enumerate(parts)]))
    if weighted:
        assert np.array_equal(gw, np.concatenate([p[4] for p in parts]))
    # every ego's PageRank from the packed graph in one call
    out, its, _ = g.pagerank_graphs(off, directed=directed, weighted=weighted, tol=1e-11)
    for k, p in enumerate(parts):
        og = O.Graph(len(p[0]), p[2], p[3], p[4], directed)
        ref = og.pagerank(directed=directed, weighted=weighted, tol=1e-11)
        assert np.abs(out[off[k]:off[k + 1]] - ref).sum() <= 1e-12, k
        assert its[k] == og.last_iters, k


def test_frame_egos_edge_cases():
    # egos without members, a table with no egos at all, labels outside the
    # range, rows whose target is in another ego
    src = np.array([0, 1, 2, 3, 0])
    tgt = np.array([1, 0, 3, 0, 0])
    node_ego = np.array([2, 2, 0, 0])
    edge_ego = np.array([2, 2, 0, 0, 7])
    g, off, ids, rows = K.frame_egos(4, src, tgt, node_ego, edge_ego, 4)
    assert off.tolist() == [0, 2, 2, 4, 4]
    assert ids.tolist() == [2, 3, 0, 1] and rows.tolist() == [2, 0, 1]
    gs, gt, _ = g.edges()
    assert gs.tolist() == [0, 2, 3] and gt.tolist() == [1, 3, 2]
    g, off, ids, rows = K.frame_egos(4, src, tgt, np.full(4, -1), None, 0)
    assert off.tolist() == [0] and g.n == 0 and g.m == 0
    g, off, ids, rows = K.frame_egos(4, src, tgt, np.full(4, -1), None, 3)
    assert off.tolist() == [0, 0, 0, 0] and g.m == 0


def test_frame_errors_follow_from_edges():
    # graph.rs:162-192 as the observed rows see it: weights first, edges
    # numbered among the observed rows
    src, tgt = np.array([0, 5, 1, 2]), np.array([1, 1, 7, 0])
    miss = np.array([0, 1, 0, 0], dtype=bool)
    msg = r"edge 1 refers to node index 7, but valid indices are 0\.\.3"
    with pytest.raises(K.EngineError, match=msg):
        K.frame_graph(3, src, tgt, None, miss)
    with pytest.raises(O.OracleError, match=msg):
        O.frame_graph_of(3, src, tgt, None, miss)
    with pytest.raises(K.EngineError, match=msg):
        K.frame_egos(3, src, tgt, np.zeros(3), None, 1, None, miss)
    w = np.array([1.0, 2.0, 3.0, np.inf])
    with pytest.raises(K.EngineError, match="edge 2 has a missing, NaN, or infinite weight"):
        K.frame_graph(3, src, tgt, w, miss)
    neg = np.array([-1, 0])
    with pytest.raises(K.EngineError, match="edge 0 refers to node index -1"):
        K.frame_graph(2, neg, np.array([1, 1]))
