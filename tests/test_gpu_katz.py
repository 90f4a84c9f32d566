"""Katz and Bonacich power centrality on the device against the CPU oracle,
through the C ABI (the reference golden vectors run in test_gpu_parity).

Bars: the reference's hand values; on R-MAT graphs, every mode, weighted
and not, within 1e-10 of the oracle relative to the largest score (the two
stop on the same rule; their sums differ only by rounding); the dense
Bonacich solve within 1e-9; the reference's errors.
"""
from __future__ import annotations

import numpy as np
import pytest

import knappnet_b200 as K
from oracle import oracle as O
from test_oracle import katz_bonacich_known_answers

pytestmark = pytest.mark.gpu


def pair(scale, weighted, seed, symmetrize=False):
    kg = K.generate_rmat(scale, 16, seed=seed, clean=True, symmetrize=symmetrize,
                         lognormal=weighted, wseed=seed + 1)
    s, t, w = kg.edges()
    return kg, O.Graph(kg.n, s, t, w, not symmetrize)


def close(a, b, rel):
    return np.abs(a - b).max() <= rel * max(np.abs(b).max(), 1e-300)


def test_known_answers():
    katz_bonacich_known_answers(K.Graph, K.EngineError)


@pytest.mark.parametrize("weighted", [False, True])
def test_katz_rmat_every_mode(weighted):
    kg, og = pair(12, weighted, 31)
    for mode in (1, 2, 3):
        _, lam, _ = og.eigenvector(mode=mode, weighted=weighted, loops=1)
        for frac, beta, normalized in ((0.5, 1.0, True), (0.9, None, False)):
            b = 1.0 if beta is not None else np.arange(kg.n) % 3 + 1.0
            a = kg.katz(alpha=frac / lam, beta=b, mode=mode, weighted=weighted, loops=1,
                        normalized=normalized)
            r = og.katz(alpha=frac / lam, beta=b, mode=mode, weighted=weighted, loops=1,
                        normalized=normalized)
            assert close(a, r, 1e-10), (mode, frac)


def test_katz_undirected_and_errors():
    kg, og = pair(11, True, 7, symmetrize=True)
    _, lam, _ = og.eigenvector(mode=3, loops=0)
    for loops in (0, 1, 2):
        a = kg.katz(alpha=0.5 / lam, loops=loops)
        r = og.katz(alpha=0.5 / lam, loops=loops)
        assert close(a, r, 1e-10), loops
    with pytest.raises(K.EngineError, match="lambda_max"):
        kg.katz(alpha=1.5 / lam, loops=0)
    with pytest.raises(K.EngineError, match="no edge weights"):
        K.Graph(3, [0, 1], [1, 2], None, True).katz(weighted=True)
    with pytest.raises(K.EngineError, match="negative weight"):
        K.Graph(3, [0, 1], [1, 2], [1.0, -1.0], True).katz(weighted=True)
    with pytest.raises(K.EngineError, match="unknown degree mode"):
        kg.katz(mode=4)


@pytest.mark.parametrize("weighted", [False, True])
def test_bonacich_rmat_series(weighted):
    kg, og = pair(12, weighted, 41)
    for mode in (1, 2, 3):
        _, lam, _ = og.eigenvector(mode=2 if mode == 1 else mode, weighted=weighted, loops=2)
        for frac in (0.5, -0.5):
            for rescale in (False, True):
                a = kg.bonacich(exponent=frac / lam, mode=mode, weighted=weighted,
                                rescale=rescale)
                r = og.bonacich(exponent=frac / lam, mode=mode, weighted=weighted,
                                rescale=rescale)
                assert not og.last_dense
                assert close(a, r, 1e-10), (mode, frac, rescale)


def test_bonacich_dense_solve():
    # exponent 1 far beyond 1 / lambda_max: the dense solve (2,000 nodes)
    s, t = K.generate_gnm(2000, 8000, False, False, seed=5)
    kg = K.Graph(2000, s, t, None, False)
    og = O.Graph(2000, s, t, None, False)
    r = og.bonacich(exponent=1.0)
    assert og.last_dense
    a = kg.bonacich(exponent=1.0)
    assert close(a, r, 1e-9)
    # singular: exponent the reciprocal of an eigenvalue (a 4-cycle has 2)
    c4 = K.Graph(4, [0, 1, 2, 3], [1, 2, 3, 0], None, False)
    with pytest.raises(K.EngineError, match="singular"):
        c4.bonacich(exponent=0.5)


def test_katz_rmat20_fixed_point():
    """Scale 20, directed: x = beta + alpha A_in x to the series tolerance."""
    import scipy.sparse as sp
    kg = K.generate_rmat(20, 16, seed=20240611, clean=True)
    _, info = kg.eigenvector_ex(mode=2, loops=1)
    alpha = 0.5 / info.eigenvalue
    x = kg.katz(alpha=alpha, normalized=False)
    off, cols, _ = kg.csr(1)
    A = sp.csr_matrix((np.ones(len(cols)), cols.astype(np.int32), off.astype(np.int64)),
                      shape=(kg.n, kg.n))
    res = np.abs(x - (1.0 + alpha * (A @ x))).max()
    assert res <= 1e-10 * np.abs(x).max(), res
    kg.close()


# ------------------------------------------------------------------ HITS
def test_hits_known_answers():
    from test_oracle import hits_known_answers
    hits_known_answers(K.Graph)


@pytest.mark.parametrize("weighted,symmetrize", [(False, False), (True, False), (True, True)])
def test_hits_rmat_matches_oracle(weighted, symmetrize):
    kg, og = pair(12, weighted, 51, symmetrize=symmetrize)
    for loops in (0, 1, 2):
        for scale in (0, 1, 2):
            a = kg.hits(weighted=weighted, loops=loops, scale=scale)
            b = og.hits(weighted=weighted, loops=loops, scale=scale)
            assert abs(a[2] - b[2]) <= 1e-9 * b[2]
            assert a[3] == b[3]
            assert close(a[0], b[0], 1e-8) and close(a[1], b[1], 1e-8), (loops, scale)


def test_hits_rmat20_singular_vector_equation():
    """Scale 20, directed: A^T A a = value a, hubs proportional to A a."""
    import scipy.sparse as sp
    kg = K.generate_rmat(20, 16, seed=20240612, clean=True)
    hubs, auths, value, unique = kg.hits(scale=2)
    off, cols, _ = kg.csr(0)
    A = sp.csr_matrix((np.ones(len(cols)), cols.astype(np.int32), off.astype(np.int64)),
                      shape=(kg.n, kg.n))
    ata = A.T @ (A @ auths)
    assert unique
    assert np.abs(ata - value * auths).max() <= 1e-8 * value * np.abs(auths).max()
    h = A @ auths
    assert np.abs(hubs - h / np.linalg.norm(h)).max() <= 1e-12
    kg.close()
