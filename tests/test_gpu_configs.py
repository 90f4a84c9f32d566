"""Parity with the CPU oracle at the benchmark configurations themselves, on
the same inputs the benchmark uses:

- C1: PageRank, FP64, on the undirected G(n = 10,000, m = 50,000), tol 1e-12:
  L1 <= 1e-12 against the oracle and the same iteration count;
- C2: eigenvector centrality by Lanczos on the symmetrised R-MAT scale 20
  graph, tol 1e-10, FP64 products and FP32 products with FP64
  reorthogonalisation: eigenvalue within 1e-9 relative, scores within 1e-8
  (max norm) of the oracle;
- C3: directed weighted PageRank on R-MAT scale 24 (lognormal FP32
  strengths), tol 1e-9: the all-FP64 path within 1e-12 L1 of the oracle
  (plus the oracle's own normalisation residual) with the same sweep count,
  and the mixed path (FP32 sweeps, FP64 anchor, refinement sweeps) within
  1e-9 L1 with the same top-100 order; for the merge-path sweep and for the
  sliced sweep (the default);
- C4a: batched personalised PageRank on R-MAT scale 22 with 256 teleport
  vectors of 1-64 seed nodes: sampled columns within 1e-9 L1 of their own
  oracle calls.

The oracle restates the reference's CPU algorithm (metrics/spectral.rs:211-281,
metrics/eigenvector.rs:746-878); the graphs are generated on the device from
the benchmark's seeds and handed to the oracle edge for edge.
"""
from __future__ import annotations

import numpy as np
import pytest

import knappnet_b200 as K
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("small_edges", [-1, 0])
def test_c1_er_10k_fp64_matches_oracle(small_edges):
    """C1 on both paths: the default one launch of the packed-graph kernel
    (the graph split over a cluster) and, with tuning key 17 at 0, the sweep
    kernels."""
    s, t = K.generate_gnm(10_000, 50_000, False, False, seed=20240701)
    g = K.Graph(10_000, s, t, None, False)
    og = O.Graph(10_000, s, t, None, False)
    ref = og.pagerank(tol=1e-12)
    try:
        if small_edges >= 0:
            K.set_tuning(K.TUNE_SMALL_EDGES, small_edges)
        x, info = g.pagerank_ex(tol=1e-12, precision=K.PREC_FP64)
    finally:
        K.set_tuning(K.TUNE_SMALL_EDGES, 1 << 18)
    assert np.abs(x - ref).sum() <= 1e-12
    assert info.iterations == og.last_iters
    assert 0 < info.change <= 1e-12
    assert (info.sweep_kernel == 0) == (small_edges < 0)
    g.close()


@pytest.fixture(scope="module")
def c2_graph():
    g = K.generate_rmat(20, 16, seed=20240702, clean=True, symmetrize=True)
    s, t, _ = g.edges()
    og = O.Graph(g.n, s, t, None, False)
    ox, olam, _ = og.eigenvector(mode=3, tol=1e-10)
    yield g, ox, olam
    g.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_c2_rmat20_lanczos_matches_oracle(c2_graph, precision):
    g, ox, olam = c2_graph
    x, info = g.eigenvector_ex(mode=3, tol=1e-10, precision=precision)
    assert abs(info.eigenvalue - olam) <= 1e-9 * olam
    assert np.abs(x - ox).max() <= 1e-8


@pytest.fixture(scope="module")
def c3_graph():
    g = K.generate_rmat(24, 16, 0.57, 0.19, 0.19, seed=20240601, clean=True,
                        lognormal=True, wseed=20240602)
    s, t, w = g.edges()
    og = O.Graph(g.n, s, t, w, True)
    del s, t, w
    ref = og.pagerank(weighted=True, tol=1e-9)
    iters = og.last_iters
    del og
    yield g, ref, iters
    g.close()


@pytest.mark.parametrize("variant", [K.VARIANT_WARP_L1, 0])
def test_c3_rmat24_fp64_and_mixed_match_oracle(c3_graph, variant):
    g, ref, iters = c3_graph
    try:
        K.set_tuning(K.TUNE_VARIANT, variant)
        x64, i64 = g.pagerank_ex(weighted=True, tol=1e-9, precision=K.PREC_FP64)
        xm, im = g.pagerank_ex(weighted=True, tol=1e-9, precision=K.PREC_MIXED)
    finally:
        K.set_tuning(K.TUNE_VARIANT, 0)
    # The oracle divides by a sequential sum of 16.8M values; allow its own
    # normalisation residual on top of the 1e-12 bar.
    resid = abs(ref.sum() - 1.0)
    assert np.abs(x64 - ref).sum() <= 1e-12 + resid
    assert i64.iterations == iters
    assert np.abs(xm - ref).sum() <= 1e-9
    top = np.argsort(-ref, kind="stable")[:100]
    assert np.array_equal(np.argsort(-xm, kind="stable")[:100], top)
    assert np.array_equal(np.argsort(-x64, kind="stable")[:100], top)


def test_c4a_rmat22_batch_columns_match_oracle():
    g = K.generate_rmat(22, 16, seed=20240703, clean=True)
    n, B = g.n, 256
    rng = np.random.default_rng(20240704)
    P = np.zeros((B, n))
    for b in range(B):
        k = int(rng.integers(1, 65))
        P[b, rng.choice(n, size=k, replace=False)] = 1.0 / k
    out, _ = g.pagerank_batch(P, precision=K.PREC_MIXED, tol=1e-10)
    s, t, _ = g.edges()
    og = O.Graph(n, s, t, None, True)
    for b in (0, 1, 128, 255):
        ref = og.pagerank(personalization=P[b], tol=1e-10)
        assert np.abs(out[b] - ref).sum() <= 1e-9, b
    g.close()
