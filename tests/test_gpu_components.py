"""Weak and strong components on the device (net_components) against the
oracle's union-find and Tarjan's algorithm (crates/engine/src/metrics/
topography.rs:183-286): labels and counts bit-exact, on random graphs, on
shapes that stress the rounds of trimming and colouring (long paths either
way, a long cycle, chains of cycles, a cycle reached only through a long
tail), and on R-MAT graphs; and eigenvector centralization (net_centralization,
topography.rs:475-498) against the oracle's restatement.
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
