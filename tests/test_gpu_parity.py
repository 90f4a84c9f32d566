"""Parity of the CUDA library with the CPU oracle and the reference's golden
files, through the C ABI.

Bars: integer CSR structure (offsets, targets, arc order) and degree counts
bit-exact; FP64 PageRank within 1e-12 L1 of the oracle; mixed-precision
PageRank within 1e-9 L1 with the same top-100 order; eigenvector centrality
within the golden tolerance (rel 1e-8 / abs 1e-9) and within 1e-9 (max
norm) of the oracle.
"""
from __future__ import annotations

import numpy as np
import pytest

import goldens
import knappnet_b200 as K
from oracle import oracle as O
from test_oracle import SplitMix64, dense, random_case

pytestmark = pytest.mark.gpu

DOC = goldens.load()


def both(fx):
    return goldens.make_graph(K.Graph, fx), goldens.make_graph(O.Graph, fx)


# ------------------------------------------------------------------ golden files
@pytest.mark.parametrize("fx_name,variant,orc", goldens.cases())
def test_golden(fx_name, variant, orc):
    fx = DOC["fixtures"][fx_name]
    g = goldens.make_graph(K.Graph, fx)
    got = goldens.run_variant(g, fx, variant)
    ok, msg = goldens.agree_variant(got, DOC["golden"][fx_name][variant][orc], variant)
    assert ok, msg


PAGERANK_CASES = [c for c in goldens.cases() if c[1].startswith("pagerank")]


@pytest.mark.parametrize("fx_name,variant,orc", PAGERANK_CASES)
def test_golden_pagerank_on_the_sweep_path(fx_name, variant, orc):
    """The PageRank golden vectors again with small graphs kept on the sweep
    kernels (tuning key 17 at 0) instead of the one-launch packed path."""
    fx = DOC["fixtures"][fx_name]
    g = goldens.make_graph(K.Graph, fx)
    try:
        K.set_tuning(K.TUNE_SMALL_EDGES, 0)
        got = goldens.run_variant(g, fx, variant)
    finally:
        K.set_tuning(K.TUNE_SMALL_EDGES, 1 << 18)
    ok, msg = goldens.agree_variant(got, DOC["golden"][fx_name][variant][orc], variant)
    assert ok, msg


# ------------------------------------------------------------------ CSR and degree
def random_graphs(seed, count, max_n):
    rng = SplitMix64(seed)
    for _ in range(count):
        n, src, tgt, w, directed = random_case(rng, max_n)
        yield n, src, tgt, w, directed


def assert_same_csr(kg, og, which):
    ko, kt, kw = kg.csr(which)
    oo, ot, ow = og.csr(which)
    assert np.array_equal(ko.astype(np.uint64), oo)
    assert np.array_equal(kt, ot)
    if ow is not None:
        assert np.array_equal(kw, ow)


@pytest.mark.parametrize("fx_name", sorted(DOC["fixtures"]))
def test_csr_bit_exact_fixtures(fx_name):
    kg, og = both(DOC["fixtures"][fx_name])
    assert_same_csr(kg, og, 0)
    if kg.directed:
        assert_same_csr(kg, og, 1)


def test_csr_bit_exact_random_multigraphs():
    for n, src, tgt, w, directed in random_graphs(7, 60, 60):
        kg = K.Graph(n, src, tgt, w, directed)
        og = O.Graph(n, src, tgt, w, directed)
        assert_same_csr(kg, og, 0)
        if directed:
            assert_same_csr(kg, og, 1)
            # directions ignored: the reference rebuilds an undirected graph
            ug = O.Graph(n, src, tgt, w, False)
            ko, kt, kw = kg.csr(2)
            oo, ot, ow = ug.csr(0)
            assert np.array_equal(ko.astype(np.uint64), oo) and np.array_equal(kt, ot)
            assert np.array_equal(kw, ow)


def test_csr_bit_exact_large_with_parallel_arcs():
    rng = np.random.default_rng(5)
    n, m = 20_000, 400_000
    src = rng.integers(0, n // 10, m)  # many parallel arcs and loops
    tgt = rng.integers(0, n // 10, m)
    w = rng.random(m)
    for directed in (True, False):
        kg = K.Graph(n, src, tgt, w, directed)
        og = O.Graph(n, src, tgt, w, directed)
        assert_same_csr(kg, og, 0)
        if directed:
            assert_same_csr(kg, og, 1)


@pytest.mark.parametrize("fx_name", sorted(DOC["fixtures"]))
def test_degree_bit_exact(fx_name):
    fx = DOC["fixtures"][fx_name]
    kg, og = both(fx)
    for mode in (1, 2, 3):
        for loops in (False, True):
            for weighted in ((False, True) if fx["weighted"] else (False,)):
                a = kg.degree(mode, loops, weighted)
                b = og.degree(mode, loops, weighted)
                if weighted:
                    assert np.allclose(a, b, rtol=1e-15, atol=0)
                else:
                    assert np.array_equal(a, b)


# ------------------------------------------------------------------ PageRank
PR_OPTIONS = [
    dict(),
    dict(loops=1),
    dict(loops=2),
    dict(directed=False),
    dict(dangling=1, pers="mod3plus1"),
    dict(pers="mod3plus1"),
    dict(damping=0.6),
]


@pytest.mark.parametrize("small_edges", [1 << 18, 0])
@pytest.mark.parametrize("fx_name", sorted(DOC["fixtures"]))
def test_pagerank_fp64_within_1e12_of_oracle(fx_name, small_edges):
    """Every fixture and option set, with FP64 solves as one packed launch
    (the default for small graphs) and on the sweep kernels (key 17 at 0)."""
    fx = DOC["fixtures"][fx_name]
    kg, og = both(fx)
    n = fx["n"]
    try:
        K.set_tuning(K.TUNE_SMALL_EDGES, small_edges)
        for opt in PR_OPTIONS + ([dict(weighted=True)] if fx["weighted"] else []):
            o = dict(opt)
            pers = o.pop("pers", None)
            p = np.asarray(goldens.node_rule(pers, n)) if pers else None
            a, ia = kg.pagerank_ex(personalization=p, **o)
            b = og.pagerank(personalization=p, **o)
            assert np.abs(a - b).sum() <= 1e-12, (opt, np.abs(a - b).sum())
            assert ia.iterations == og.last_iters, opt
    finally:
        K.set_tuning(K.TUNE_SMALL_EDGES, 1 << 18)


def test_pagerank_reference_signature_call():
    g = K.Graph(5, [0, 0, 1, 2, 3, 2], [1, 2, 2, 0, 2, 4], None, True)
    a = g.pagerank_reference_call(0.85, 1, 0, None, 0, 0, 0.0, 0, 4)
    want = [0.2142011097, 0.1574496602, 0.3477339318, 0.0664141886, 0.2142011097]
    assert np.allclose(a, want, atol=1e-9, rtol=0)


def test_pagerank_hand_values():
    g = K.Graph(5, [0, 0, 1, 2, 3, 2], [1, 2, 2, 0, 2, 4], None, True)
    p = [1.0, 0.0, 0.0, 0.0, 0.0]
    assert np.allclose(g.pagerank(personalization=p),
                       [0.3928645968, 0.1669674536, 0.3088897892, 0.0, 0.1312781604],
                       atol=1e-9, rtol=0)
    assert np.allclose(g.pagerank(personalization=p, dangling=1),
                       [0.3166510816, 0.1629073936, 0.3254597594, 0.0283306839, 0.1666510816],
                       atol=1e-9, rtol=0)


def test_pagerank_stationary_random_cases():
    rng = SplitMix64(21)
    for _ in range(60):
        n, src, tgt, w, directed = random_case(rng, 30)
        weighted = rng.below(2) == 0
        g = K.Graph(n, src, tgt, w if weighted else None, directed)
        x = g.pagerank(weighted=weighted)
        assert abs(x.sum() - 1.0) < 1e-12
        a = dense(n, src, tgt, w, directed, weighted, False, 2.0)
        out = a.sum(axis=1)
        stuck = x[out == 0].sum()
        flow = np.array([sum(a[j, i] / out[j] * x[j] for j in range(n) if out[j] > 0)
                         for i in range(n)])
        rhs = 0.85 * (flow + stuck / n) + 0.15 / n
        assert np.abs(x - rhs).max() < 1e-10


def rmat_pair(scale, weighted, symmetrize=False, seed=3):
    kg = K.generate_rmat(scale, 16, seed=seed, clean=True, symmetrize=symmetrize,
                         lognormal=weighted, wseed=seed + 100)
    s, t, w = kg.edges()
    og = O.Graph(kg.n, s, t, w, not symmetrize)
    return kg, og


# refine 1 (default): after the FP32 sweeps, one FP64 anchor sweep and
# refinement sweeps gathering the FP32 correction; refine 0: FP64 sweeps.
@pytest.mark.parametrize("weighted,refine", [(False, 1), (True, 1), (True, 0)])
def test_pagerank_rmat_fp64_and_mixed(weighted, refine):
    kg, og = rmat_pair(14, weighted)
    ref = og.pagerank(weighted=weighted, tol=1e-9)
    x64, i64 = kg.pagerank_ex(weighted=weighted, tol=1e-9, precision=K.PREC_FP64)
    assert np.abs(x64 - ref).sum() <= 1e-12
    assert i64.iterations == og.last_iters
    try:  # the same FP64 solve on the sweep kernels rather than one packed launch
        K.set_tuning(K.TUNE_SMALL_EDGES, 0)
        s64, j64 = kg.pagerank_ex(weighted=weighted, tol=1e-9, precision=K.PREC_FP64)
    finally:
        K.set_tuning(K.TUNE_SMALL_EDGES, 1 << 18)
    assert j64.sweep_kernel != 0
    assert np.abs(s64 - ref).sum() <= 1e-12
    assert j64.iterations == og.last_iters
    try:
        K.set_tuning(K.TUNE_REFINE, refine)
        xm, im = kg.pagerank_ex(weighted=weighted, tol=1e-9, precision=K.PREC_MIXED)
    finally:
        K.set_tuning(K.TUNE_REFINE, 1)
    assert np.abs(xm - ref).sum() <= 1e-9, np.abs(xm - ref).sum()
    assert im.iterations_fp32 > 0
    top = np.argsort(-ref, kind="stable")[:100]
    assert np.array_equal(np.argsort(-xm, kind="stable")[:100], top)
    # the mixed path follows the FP64 trajectory: same stopping sweep, and
    # far inside the 1e-9 bar
    assert im.iterations == i64.iterations
    assert np.abs(xm - x64).sum() <= 1e-10, np.abs(xm - x64).sum()


def test_pagerank_personalized_and_undirected_rmat():
    kg, og = rmat_pair(12, True)
    n = kg.n
    p = np.zeros(n)
    p[[3, 17, 400]] = [1.0, 2.0, 0.5]
    for opts in (dict(personalization=p), dict(personalization=p, dangling=1),
                 dict(directed=False), dict(directed=False, loops=1)):
        a = kg.pagerank(weighted=True, **opts)
        b = og.pagerank(weighted=True, **opts)
        assert np.abs(a - b).sum() <= 1e-12, opts


def test_pagerank_repeat_runs_are_bit_identical():
    kg, _ = rmat_pair(13, True)
    a = kg.pagerank(weighted=True)
    b = kg.pagerank(weighted=True)
    assert np.array_equal(a, b)


def test_pagerank_errors():
    g = K.Graph(5, [0, 0, 1, 2, 3, 2], [1, 2, 2, 0, 2, 4], None, True)
    with pytest.raises(K.EngineError, match="damping is 1.5"):
        g.pagerank(damping=1.5)
    with pytest.raises(K.EngineError, match="dangling-node code 7"):
        g.pagerank(dangling=7)
    with pytest.raises(K.EngineError, match="self-loop weight code 5"):
        g.pagerank(loops=5)
    with pytest.raises(K.EngineError, match="no edge weights"):
        g.pagerank(weighted=True)
    with pytest.raises(K.EngineError, match="finite, nonnegative"):
        g.pagerank(personalization=[1.0, -1.0, 0, 0, 0])
    with pytest.raises(K.EngineError, match="positive sum"):
        g.pagerank(personalization=[0.0] * 5)
    with pytest.raises(K.EngineError, match="did not converge"):
        g.pagerank(tol=1e-15, max_iter=2)
    neg = K.Graph(3, [0, 1], [1, 2], [1.0, -2.0], True)
    with pytest.raises(K.EngineError, match="edge 1 has negative weight -2"):
        neg.pagerank(weighted=True)
    with pytest.raises(K.EngineError, match="edge 1 refers to node index 9"):
        K.Graph(3, [0, 1], [1, 9], None, True)
    with pytest.raises(K.EngineError, match="edge 0 refers to node index -1"):
        K.Graph(3, [-1, 1], [1, 9], None, True)
    with pytest.raises(K.EngineError, match="NaN"):
        K.Graph(3, [0, 1], [1, 2], [1.0, float("nan")], True)


def test_empty_and_single_node():
    e = K.Graph(0, [], [], None, True)
    assert e.pagerank().size == 0
    s = K.Graph(1, [], [], None, True)
    assert np.allclose(s.pagerank(), [1.0])


# ------------------------------------------------------------------ eigenvector
def test_eigen_closed_forms():
    star = K.Graph(5, [0, 0, 0, 0], [1, 2, 3, 4], None, False)
    v, lam, conn = star.eigenvector()
    assert abs(lam - 2.0) < 1e-10 and conn
    assert np.allclose(v, [1.0, 0.5, 0.5, 0.5, 0.5], atol=1e-10, rtol=0)
    path = K.Graph(4, [0, 1, 2], [1, 2, 3], None, False)
    v, lam, _ = path.eigenvector()
    phi = (1 + 5 ** 0.5) / 2
    assert abs(lam - phi) < 1e-10
    assert np.allclose(v, [1 / phi, 1, 1, 1 / phi], atol=1e-10, rtol=0)
    lw = K.Graph(2, [0, 0], [0, 1], [1.0, 3.0], False)
    assert abs(lw.eigenvector()[1] - (1 + 2 ** 0.5)) < 1e-10
    assert abs(lw.eigenvector(loops=1, weighted=True)[1] - (1 + 37 ** 0.5) / 2) < 1e-10
    empty = K.Graph(3, [], [], None, False)
    v, lam, conn = empty.eigenvector()
    assert v.tolist() == [1.0, 1.0, 1.0] and lam == 0.0 and not conn
    dag = K.Graph(3, [0, 1], [1, 2], None, True)
    assert dag.eigenvector(mode=2)[0].tolist() == [0.0, 0.0, 1.0]
    assert dag.eigenvector(mode=1)[0].tolist() == [1.0, 0.0, 0.0]
    tri = K.Graph(5, [0, 1, 2, 3], [1, 2, 0, 4], None, False)
    v, lam, conn = tri.eigenvector()
    assert not conn and abs(lam - 2.0) < 1e-10
    assert np.allclose(v, [1, 1, 1, 0, 0], atol=1e-9, rtol=0)


def test_eigen_directed_modes():
    g = K.Graph(3, [0, 1, 2, 2], [1, 2, 0, 1], None, True)
    ins, li, _ = g.eigenvector(mode=2)
    outs, lo, _ = g.eigenvector(mode=1)
    a = np.array([[0.0, 1, 0], [0, 0, 1], [1, 1, 0]])
    assert np.allclose(a.T @ ins, li * ins, atol=1e-10)
    assert np.allclose(a @ outs, lo * outs, atol=1e-10)


@pytest.mark.parametrize("fx_name", sorted(DOC["fixtures"]))
def test_eigen_matches_oracle_on_fixtures(fx_name):
    fx = DOC["fixtures"][fx_name]
    kg, og = both(fx)
    for opts in (dict(), dict(mode=1), dict(mode=3), dict(scale=1, loops=1)):
        try:
            b = og.eigenvector(**opts)
        except O.OracleError:
            with pytest.raises(K.EngineError):
                kg.eigenvector(**opts)
            continue
        a = kg.eigenvector(**opts)
        assert np.abs(a[0] - b[0]).max() <= 1e-9, opts
        assert abs(a[1] - b[1]) <= 1e-9 * max(1.0, abs(b[1])), opts
        assert a[2] == b[2]


def test_lanczos_eigen_equation_random():
    rng = SplitMix64(11)
    for _ in range(40):
        n, src, tgt, w, _ = random_case(rng, 40)
        weighted = rng.below(2) == 0
        g = K.Graph(n, src, tgt, w if weighted else None, False)
        x, lam, _ = g.eigenvector(weighted=weighted, scale=1)
        if lam == 0.0:
            continue
        a = dense(n, src, tgt, w, False, weighted, True, 2.0)
        assert (x >= 0).all()
        assert np.all(np.abs(a @ x - lam * x) <= 1e-9 * (1 + lam))


@pytest.mark.parametrize("precision", [0, 1])
def test_lanczos_symmetric_rmat_matches_oracle(precision):
    kg, og = rmat_pair(13, False, symmetrize=True)
    b, lb, cb = og.eigenvector(mode=3, tol=1e-10)
    a, info = kg.eigenvector_ex(mode=3, tol=1e-10, precision=precision)
    assert abs(info.eigenvalue - lb) <= 1e-9 * lb
    assert np.abs(a - b).max() <= 1e-8
    assert bool(info.connected) == cb


def projected_cases():
    """Symmetric matrices like the Lanczos process's projected ones: random,
    tridiagonal, arrowhead (after a thick restart), with a cluster of close
    eigenvalues, diagonal, of every order from 1 to 20."""
    rng = np.random.default_rng(11)
    for n in range(1, 21):
        a = rng.standard_normal((n, n))
        yield "random", (a + a.T) / 2
        off = rng.random(n - 1)
        yield "tridiagonal", np.diag(rng.random(n) * 10) + np.diag(off, 1) + np.diag(off, -1)
        h = np.diag(np.sort(rng.random(n))[::-1] * 50)
        if n > 2:
            p = min(8, n - 1)
            h[:p, p] = h[p, :p] = rng.standard_normal(p)
        yield "arrowhead", h
    q, _ = np.linalg.qr(rng.standard_normal((12, 12)))
    yield "cluster", q @ np.diag([5.0, 5.0 + 1e-12, 5.0 + 2e-12] + list(range(9))) @ q.T
    yield "diagonal", np.diag([3.0, 1.0, 2.0, 1.0])


def test_projected_eigensolver_on_device_matches_eispack():
    """The warp solver Lanczos uses for its projected matrices against the
    oracle's EISPACK restatement (crates/engine/src/linalg.rs:478-720):
    eigenvalues within 1e-13 of the largest, eigenvectors the same up to
    rounding where eigenvalues are apart, and A V = V diag(d) for all."""
    for kind, a in projected_cases():
        d, v = K.projected_eigen(a)
        od, ov = O.symmetric_eigen(a)
        scale = max(1.0, np.abs(od).max())
        assert np.abs(d - od).max() <= 1e-13 * scale, kind
        assert np.abs(a @ v - v * d).max() <= 1e-12 * scale, kind
        assert np.abs(v.T @ v - np.eye(len(d))).max() <= 1e-12, kind
        gaps = np.diff(od)
        if kind != "cluster" and (len(od) < 2 or gaps.min() > 1e-6 * scale):
            assert np.abs(v - ov).max() <= 1e-10, kind


def test_power_iteration_directed_rmat_matches_oracle():
    kg, og = rmat_pair(11, True, seed=9)
    for mode in (1, 2):
        try:
            b = og.eigenvector(mode=mode, weighted=True, tol=1e-10)
        except O.OracleError:
            continue
        a = kg.eigenvector(mode=mode, weighted=True, tol=1e-10)
        assert np.abs(a[0] - b[0]).max() <= 1e-9
        assert abs(a[1] - b[1]) <= 1e-9 * max(1.0, b[1])


# ------------------------------------------------------------------ generator
def test_rmat_generator_matches_oracle():
    scale, ef, seed = 10, 16, 77
    raw = K.generate_rmat(scale, ef, seed=seed, clean=False)
    s, t, _ = raw.edges()
    os_, ot = O.rmat_raw(scale, ef << scale, 0.57, 0.19, 0.19, seed)
    assert np.array_equal(s, os_) and np.array_equal(t, ot)
    clean = K.generate_rmat(scale, ef, seed=seed, clean=True)
    cs, ct, _ = clean.edges()
    keep = os_ != ot
    key = np.unique(os_[keep].astype(np.int64) << scale | ot[keep].astype(np.int64))
    assert np.array_equal(cs, key >> scale) and np.array_equal(ct, key & ((1 << scale) - 1))
    sym = K.generate_rmat(scale, ef, seed=seed, symmetrize=True)
    ss, st, _ = sym.edges()
    lo, hi = np.minimum(os_, ot)[keep], np.maximum(os_, ot)[keep]
    key = np.unique(lo.astype(np.int64) << scale | hi.astype(np.int64))
    assert np.array_equal(ss, key >> scale) and np.array_equal(st, key & ((1 << scale) - 1))
    assert not sym.directed


def test_lognormal_weights_match_box_muller():
    g = K.generate_rmat(8, 8, seed=1, lognormal=True, wseed=5)
    _, _, w = g.edges()
    u = np.array([O.stream_u32(5, e, 4) for e in range(len(w))], dtype=np.uint64)
    a = (u[:, 0] << np.uint64(32) | u[:, 1]) >> np.uint64(11)
    b = (u[:, 2] << np.uint64(32) | u[:, 3]) >> np.uint64(11)
    u1 = a.astype(np.float64) / 2.0 ** 53
    u2 = b.astype(np.float64) / 2.0 ** 53
    z = np.sqrt(-2 * np.log(1 - u1)) * np.cos(2 * np.pi * u2)
    want = np.exp(z).astype(np.float32).astype(np.float64)
    assert np.abs(w / want - 1).max() <= 2 ** -23
    assert abs(np.log(w).mean()) < 0.1 and abs(np.log(w).std() - 1) < 0.1


# Variants 6 and 7 keep the most gathered nodes in shared memory: a cap of
# 1000 nodes splits the scale-12 graph's gathers between shared memory and
# global memory, 0 sends all of them to global memory, -1 (no cap) holds the
# whole iterate; relabel 0 falls back to the plain warp kernel. Warp-tile
# variants (2-4, 8) run on a persistent grid (persist 1, the default) or with
# one warp per tile (persist 0); variant 8 lets only gathers of columns below
# the cap allocate in L1.
@pytest.mark.parametrize("variant,ipt,relabel,hot,persist", [
    (1, 4, 0, -1, 1), (1, 8, 1, -1, 1), (2, 4, 1, -1, 1), (2, 8, 0, -1, 1), (2, 8, 1, -1, 1),
    (2, 16, 1, -1, 1), (3, 8, 1, -1, 0), (4, 8, 1, -1, 0), (4, 4, 1, -1, 1), (4, 8, 0, -1, 1),
    (6, 8, 1, -1, 1), (6, 8, 1, 1000, 1), (6, 8, 1, 0, 1), (6, 4, 1, 1000, 1),
    (6, 16, 1, 1000, 1), (7, 8, 1, 1000, 1), (7, 4, 1, 1000, 1), (6, 8, 0, -1, 1),
    (8, 8, 1, 1000, 1), (8, 4, 1, 0, 1), (8, 8, 1, 0, 0)])
def test_pagerank_sweep_variants_match_oracle(variant, ipt, relabel, hot, persist):
    kg, og = rmat_pair(12, True, seed=21)
    n = kg.n
    p = np.zeros(n)
    p[[1, 50, 600]] = 1.0
    try:
        K.set_tuning(K.TUNE_VARIANT, variant)
        K.set_tuning(K.TUNE_IPT, ipt)
        K.set_tuning(K.TUNE_RELABEL, relabel)
        K.set_tuning(K.TUNE_HOT_NODES, hot)
        K.set_tuning(K.TUNE_PERSISTENT, persist)
        for opts in (dict(), dict(personalization=p), dict(directed=False)):
            b = og.pagerank(weighted=True, **opts)
            a = kg.pagerank(weighted=True, **opts)
            assert np.abs(a - b).sum() <= 1e-12, opts
            am, _ = kg.pagerank_ex(weighted=True, precision=K.PREC_MIXED, tol=1e-10,
                                   personalization=opts.get("personalization"),
                                   directed=opts.get("directed", True))
            bm = og.pagerank(weighted=True, tol=1e-10, **opts)
            assert np.abs(am - bm).sum() <= 1e-9, opts
    finally:
        K.set_tuning(K.TUNE_VARIANT, 0)
        K.set_tuning(K.TUNE_IPT, 0)
        K.set_tuning(K.TUNE_RELABEL, 1)
        K.set_tuning(K.TUNE_HOT_NODES, -1)
        K.set_tuning(K.TUNE_PERSISTENT, 1)


@pytest.mark.parametrize("variant,long_row", [(9, 0), (9, 16), (9, 255), (9, 1), (10, 0),
                                              (10, 200), (12, 0), (12, 16), (12, 1), (12, 200)])
def test_sliced_sweep_matches_oracle(variant, long_row):
    """The sliced layout (rows renumbered by length; long rows by whole
    warps in pieces, the others one lane per row): FP64 and mixed (FP32
    sweeps, FP64 anchor, refinement) solves, every option set, against
    the oracle. Long-row thresholds from 1 (every row taken by a warp) to
    255 (the longest rows a slice holds)."""
    kg, og = rmat_pair(12, True, seed=23)
    n = kg.n
    p = np.zeros(n)
    p[[3, 70, 900]] = 1.0
    try:
        K.set_tuning(K.TUNE_VARIANT, variant)
        K.set_tuning(K.TUNE_LONG_ROW, long_row)
        for opts in (dict(), dict(personalization=p), dict(directed=False),
                     dict(personalization=p, dangling=1), dict(weighted=False)):
            o = dict(weighted=True)
            o.update(opts)
            b = og.pagerank(**o)
            a, ia = kg.pagerank_ex(precision=K.PREC_FP64, **o)
            assert np.abs(a - b).sum() <= 1e-12, opts
            assert ia.iterations == og.last_iters, opts
            bm = og.pagerank(tol=1e-10, **o)
            am, _ = kg.pagerank_ex(precision=K.PREC_MIXED, tol=1e-10, **o)
            assert np.abs(am - bm).sum() <= 1e-9, opts
            top = np.argsort(-bm, kind="stable")[:100]
            assert np.array_equal(np.argsort(-am, kind="stable")[:100], top), opts
        # repeated solves are bit-identical
        x1, _ = kg.pagerank_ex(weighted=True, precision=K.PREC_MIXED, tol=1e-10)
        x2, _ = kg.pagerank_ex(weighted=True, precision=K.PREC_MIXED, tol=1e-10)
        assert np.array_equal(x1, x2)
    finally:
        K.set_tuning(K.TUNE_VARIANT, 0)
        K.set_tuning(K.TUNE_LONG_ROW, 0)


@pytest.mark.parametrize("long_row", [0, 1, 16, 200])
def test_bulk_staged_sweep_matches_sliced_sweep(long_row):
    """Kernel 12 stages the arc streams in shared memory by bulk copies and
    adds every row's arcs in kernel 9's order; only the per-warp partials of
    the epilogue's scalars (iterate sum, dangling mass, change) associate
    differently, because the two kernels keep different numbers of warps
    resident. Every solve, in every precision, with 4 or 8 arc positions per
    chunk and 1 to 4 CTAs per SM, agrees with kernel 9 to rounding and takes
    the same number of sweeps (one more or fewer at most); repeated solves
    are bit-identical."""
    kg, _ = rmat_pair(16, True, seed=29)
    p = np.zeros(kg.n)
    p[[5, 600, 7000]] = 1.0
    runs = [(dict(precision=K.PREC_FP64), 1e-13), (dict(precision=K.PREC_MIXED, tol=1e-10), 1e-10),
            (dict(precision=K.PREC_FP32, tol=1e-6), 1e-5),
            (dict(precision=K.PREC_MIXED, tol=1e-10, personalization=p, dangling=1), 1e-10),
            (dict(precision=K.PREC_FP64, directed=False), 1e-13),
            (dict(precision=K.PREC_MIXED, weighted=False), 1e-10)]
    try:
        K.set_tuning(K.TUNE_LONG_ROW, long_row)
        for ipt in (0, 8):
            K.set_tuning(K.TUNE_IPT, ipt)
            for o, bar in runs:
                o = dict(o)
                o.setdefault("weighted", True)
                K.set_tuning(K.TUNE_VARIANT, 9)
                ref, ri = kg.pagerank_ex(**o)
                for ctas in (0, 1, 3):
                    K.set_tuning(K.TUNE_VARIANT, 12)
                    K.set_tuning(K.TUNE_BULK_CTAS, ctas)
                    got, gi = kg.pagerank_ex(**o)
                    again, _ = kg.pagerank_ex(**o)
                    assert gi.sweep_kernel == 12
                    assert np.array_equal(got, again), (ipt, o, ctas)
                    assert np.abs(got - ref).sum() <= bar, (ipt, o, ctas)
                    assert abs(gi.iterations - ri.iterations) <= 1, (ipt, o, ctas)
    finally:
        K.set_tuning(K.TUNE_VARIANT, 0)
        K.set_tuning(K.TUNE_LONG_ROW, 0)
        K.set_tuning(K.TUNE_IPT, 0)
        K.set_tuning(K.TUNE_BULK_CTAS, 0)


def test_bulk_staged_wait_runs_out_and_the_context_stays_usable():
    """Kernel 12's waits on its staged copies are bounded. With tuning key 14
    the grid's first warp never issues the copies of its first chunk, so its
    wait on that chunk's barrier runs out after about a second: the sweep
    marks its state, the solve fails with an error instead of hanging, and
    the next solve on the same handle is correct."""
    kg, og = rmat_pair(12, True, seed=31)
    ref = og.pagerank(weighted=True)
    try:
        K.set_tuning(K.TUNE_VARIANT, 12)
        K.set_tuning(K.TUNE_BULK_SKIP_CHUNK, 0)
        with pytest.raises(K.EngineError, match="gave up waiting for its staged arc copies"):
            kg.pagerank_ex(weighted=True, precision=K.PREC_FP64)
        K.set_tuning(K.TUNE_BULK_SKIP_CHUNK, -1)
        a, info = kg.pagerank_ex(weighted=True, precision=K.PREC_FP64)
        assert info.sweep_kernel == 12
        assert np.abs(a - ref).sum() <= 1e-12
        assert info.iterations == og.last_iters
    finally:
        K.set_tuning(K.TUNE_BULK_SKIP_CHUNK, -1)
        K.set_tuning(K.TUNE_VARIANT, 0)


# The sweep kernels the tuner chooses between (pagerank.cu, tuned_sweep):
# (kernel, long-row threshold, L1-allocating FP32 columns).
TUNER_CANDIDATES = [(9, 255, 49152), (9, 255, 24576), (9, 255, 98304), (10, 255, 49152),
                    (9, 64, 49152), (8, 0, 24576)]


@pytest.mark.parametrize("variant,long_row,hot", TUNER_CANDIDATES)
def test_tuner_candidates_match_oracle(variant, long_row, hot):
    """Each kernel the tuner may pick, pinned, meets the oracle bars on a
    weighted R-MAT 14: FP64 within 1e-12 L1 and the same sweep count, mixed
    within 1e-9 with the same top-100 order."""
    kg, og = rmat_pair(14, True, seed=27)
    try:
        K.set_tuning(K.TUNE_VARIANT, variant)
        K.set_tuning(K.TUNE_LONG_ROW, long_row)
        K.set_tuning(K.TUNE_HOT_NODES, hot)
        b = og.pagerank(weighted=True, tol=1e-10)
        a, ia = kg.pagerank_ex(weighted=True, tol=1e-10, precision=K.PREC_FP64)
        assert np.abs(a - b).sum() <= 1e-12
        assert ia.iterations == og.last_iters
        assert ia.sweep_kernel == variant and ia.hot_columns == hot
        am, im = kg.pagerank_ex(weighted=True, tol=1e-10, precision=K.PREC_MIXED)
        assert np.abs(am - b).sum() <= 1e-9
        top = np.argsort(-b, kind="stable")[:100]
        assert np.array_equal(np.argsort(-am, kind="stable")[:100], top)
        if variant in (9, 10):
            assert im.long_row == long_row
    finally:
        K.set_tuning(K.TUNE_VARIANT, 0)
        K.set_tuning(K.TUNE_LONG_ROW, 0)
        K.set_tuning(K.TUNE_HOT_NODES, -1)


def test_tuner_picks_once_per_operator_and_reports_it():
    """On an operator of at least 2^21 arcs the first solve times the
    candidates and keeps the fastest; later solves on the operator reuse it
    (and give bit-identical results), the pick is one of the candidates, and
    the results meet the oracle bars. With the tuner off, kernel 9."""
    kg, og = rmat_pair(18, True, seed=29)
    assert kg.csr(1)[0][-1] >= 1 << 21
    b = og.pagerank(weighted=True, tol=1e-10)
    x1, i1 = kg.pagerank_ex(weighted=True, tol=1e-10, precision=K.PREC_MIXED)
    x2, i2 = kg.pagerank_ex(weighted=True, tol=1e-10, precision=K.PREC_MIXED)
    pick = (i1.sweep_kernel, i1.long_row if i1.sweep_kernel != 8 else 0, i1.hot_columns)
    # 64 warps per SM is a candidate for FP64 solves only
    assert pick in TUNER_CANDIDATES and pick[0] != 10
    assert (i2.sweep_kernel, i2.long_row, i2.hot_columns) == \
        (i1.sweep_kernel, i1.long_row, i1.hot_columns)
    assert np.array_equal(x1, x2)
    assert np.abs(x1 - b).sum() <= 1e-9
    x64, i64 = kg.pagerank_ex(weighted=True, tol=1e-10, precision=K.PREC_FP64)
    assert (i64.sweep_kernel, i64.long_row if i64.sweep_kernel != 8 else 0,
            i64.hot_columns) in TUNER_CANDIDATES
    assert np.abs(x64 - b).sum() <= 1e-12 + abs(b.sum() - 1.0)
    assert i64.iterations == og.last_iters
    try:
        K.set_tuning(K.TUNE_AUTOTUNE, 0)
        kg2, _ = rmat_pair(18, True, seed=29)
        _, i3 = kg2.pagerank_ex(weighted=True, tol=1e-10, precision=K.PREC_MIXED)
        assert (i3.sweep_kernel, i3.long_row, i3.hot_columns) == (9, 255, 49152)
    finally:
        K.set_tuning(K.TUNE_AUTOTUNE, 1)


def test_sliced_sweep_on_fixtures_and_edge_cases():
    """Every golden fixture (empty graph, single node, loops, parallel arcs,
    disconnected parts) and every loop code through the sliced layout."""
    try:
        K.set_tuning(K.TUNE_VARIANT, 9)
        for name in sorted(DOC["fixtures"]):
            kg, og = both(DOC["fixtures"][name])
            for loops in (0, 1, 2):
                for weighted in ((False, True) if kg.weighted else (False,)):
                    b = og.pagerank(weighted=weighted, loops=loops)
                    a = kg.pagerank(weighted=weighted, loops=loops)
                    assert np.abs(a - b).sum() <= 1e-12, (name, loops, weighted)
                    am, _ = kg.pagerank_ex(weighted=weighted, loops=loops,
                                           precision=K.PREC_MIXED, tol=1e-10)
                    assert np.abs(am - og.pagerank(weighted=weighted, loops=loops,
                                                   tol=1e-10)).sum() <= 1e-9, name
    finally:
        K.set_tuning(K.TUNE_VARIANT, 0)


@pytest.mark.parametrize("variant", [6, 7])
def test_hot_node_sweep_larger_than_shared_memory(variant):
    """Scale 17 (131,072 nodes): more nodes than shared memory holds, so
    gathers split between the cached head of the iterate and global memory
    with the kernel's own capacity."""
    kg, og = rmat_pair(17, True, seed=5)
    ref = og.pagerank(weighted=True, tol=1e-10)
    try:
        K.set_tuning(K.TUNE_VARIANT, variant)
        x64, i64 = kg.pagerank_ex(weighted=True, tol=1e-10, precision=K.PREC_FP64)
        xm, _ = kg.pagerank_ex(weighted=True, tol=1e-10, precision=K.PREC_MIXED)
    finally:
        K.set_tuning(K.TUNE_VARIANT, 0)
    # The oracle, like the reference, divides by a sequential sum of the n
    # entries; adding the many identical teleport-only values one by one
    # rounds with a bias, so at 131,072 nodes its output sums to 1 + 1.4e-12
    # (the device's fixed-tree sums stay within a few ulps of 1). The bar
    # allows that residual, and the renormalised oracle answer must agree to
    # 1e-12.
    resid = abs(ref.sum() - 1.0)
    assert np.abs(x64 - ref).sum() <= 1e-12 + resid
    assert np.abs(x64 - ref / ref.sum()).sum() <= 1e-12
    assert i64.iterations == og.last_iters
    assert np.abs(xm - ref).sum() <= 1e-9
    top = np.argsort(-ref, kind="stable")[:100]
    assert np.array_equal(np.argsort(-xm, kind="stable")[:100], top)


# ------------------------------------------------------------------ batched personalised
def seed_vectors(n, B, seed):
    """B teleport vectors, each uniform over 1..64 seed nodes."""
    rng = np.random.default_rng(seed)
    P = np.zeros((B, n))
    for b in range(B):
        k = int(rng.integers(1, 65))
        P[b, rng.choice(n, size=min(k, n), replace=False)] = 1.0
    return P


@pytest.mark.parametrize("precision,B", [(0, 40), (1, 40), (0, 300), (1, 300)])
def test_pagerank_batch_matches_per_vector_oracle(precision, B):
    kg, og = rmat_pair(11 if B > 100 else 12, True, seed=31)
    P = seed_vectors(kg.n, B, 7)
    out, info = kg.pagerank_batch(P, weighted=True, precision=precision, tol=1e-10)
    assert out.shape == P.shape
    worst = 0.0
    for b in range(B):
        ref = og.pagerank(weighted=True, personalization=P[b], tol=1e-10)
        err = np.abs(out[b] - ref).sum()
        worst = max(worst, err)
        assert err <= (1e-12 if precision == 0 else 1e-9), (b, err)
    assert info.max_column_iterations >= 1


@pytest.mark.parametrize("refine", [1, 0])
def test_pagerank_batch_refinement_follows_the_fp64_trajectory(refine):
    """Mixed batches end with one FP64 anchor sweep and refinement sweeps
    gathering the FP32 correction (tuning key 9 at 1, the default) or with
    plain FP64 sweeps (0): every column within 1e-9 of its oracle solve,
    and within 5e-10 of the all-FP64 batch (a column may stop one sweep
    apart, whose change is below the 1e-10 tolerance)."""
    kg, og = rmat_pair(12, True, seed=37)
    P = seed_vectors(kg.n, 72, 11)
    x64, i64 = kg.pagerank_batch(P, weighted=True, precision=0, tol=1e-10)
    try:
        K.set_tuning(K.TUNE_REFINE, refine)
        xm, im = kg.pagerank_batch(P, weighted=True, precision=1, tol=1e-10)
        again, _ = kg.pagerank_batch(P, weighted=True, precision=1, tol=1e-10)
    finally:
        K.set_tuning(K.TUNE_REFINE, 1)
    assert im.refined == refine and i64.refined == 0
    assert im.sweeps_fp32 > 0
    assert np.array_equal(xm, again)
    for b in range(P.shape[0]):
        ref = og.pagerank(weighted=True, personalization=P[b], tol=1e-10)
        assert np.abs(xm[b] - ref).sum() <= 1e-9, b
        assert np.abs(xm[b] - x64[b]).sum() <= 5e-10, b


@pytest.mark.parametrize("precision", [0, 1])
def test_pagerank_batch_dense_teleport(precision):
    """Teleport columns with every entry positive (the dense layout; seed
    sets take the sparse one): each column matches its own oracle solve."""
    kg, og = rmat_pair(11, True, seed=33)
    rng = np.random.default_rng(34)
    P = rng.uniform(0.1, 2.0, (24, kg.n))
    P[3, ::2] = 0.0  # one column half empty
    out, _ = kg.pagerank_batch(P, weighted=True, precision=precision, tol=1e-10)
    for b in range(P.shape[0]):
        ref = og.pagerank(weighted=True, personalization=P[b], tol=1e-10)
        err = np.abs(out[b] - ref).sum()
        assert err <= (1e-12 if precision == 0 else 1e-9), (b, err)


def test_pagerank_batch_options_and_errors():
    kg, og = rmat_pair(10, True, seed=5)
    P = seed_vectors(kg.n, 5, 3)
    for opts in (dict(dangling=1), dict(directed=False), dict(loops=1, damping=0.7)):
        out, _ = kg.pagerank_batch(P, weighted=True, **opts)
        for b in range(5):
            ref = og.pagerank(weighted=True, personalization=P[b], **opts)
            assert np.abs(out[b] - ref).sum() <= 1e-12, opts
    bad = P.copy()
    bad[2, 0] = -1.0
    with pytest.raises(K.EngineError, match="nonnegative"):
        kg.pagerank_batch(bad)
    zero = P.copy()
    zero[1] = 0.0
    with pytest.raises(K.EngineError, match="positive sum"):
        kg.pagerank_batch(zero)


# ------------------------------------------------------------------ packed graphs
@pytest.mark.parametrize("directed,weighted", [(False, False), (True, True)])
def test_pagerank_graphs_matches_each_graph(directed, weighted):
    sizes = K.power_law_sizes(60, 2.1, 5, 400, seed=4)
    m = np.minimum(6 * sizes, sizes * (sizes - 1) // (1 if directed else 2))
    src, tgt = K.generate_gnm(sizes, m, directed, False, seed=12)
    off = np.concatenate([[0], np.cumsum(sizes)])
    rng = np.random.default_rng(1)
    w = rng.lognormal(size=len(src)) if weighted else None
    g = K.Graph(int(off[-1]), src, tgt, w, directed)
    out, its, info = g.pagerank_graphs(off, weighted=weighted, tol=1e-11)
    for k in range(len(sizes)):
        lo, hi = off[k], off[k + 1]
        sel = (src >= lo) & (src < hi)
        og = O.Graph(hi - lo, src[sel] - lo, tgt[sel] - lo, None if w is None else w[sel],
                     directed)
        ref = og.pagerank(weighted=weighted, tol=1e-11)
        assert np.abs(out[lo:hi] - ref).sum() <= 1e-12, k
        assert its[k] == og.last_iters, k
    assert info.kernel_launches == 1


@pytest.mark.parametrize("cluster", [4, 8])
def test_pagerank_graphs_splits_large_graphs_over_clusters(cluster):
    """Graphs of at least 50 nodes (tuning key 15) are each split over a
    thread-block cluster of 4 or 8 CTAs (key 16) that exchange their
    partial sums through distributed shared memory; every graph still
    matches its own oracle call, with the same iteration count, and repeated
    calls give the same bits."""
    sizes = K.power_law_sizes(80, 2.1, 5, 3000, seed=14)
    m = np.minimum(6 * sizes, sizes * (sizes - 1) // 2)
    src, tgt = K.generate_gnm(sizes, m, False, False, seed=15)
    off = np.concatenate([[0], np.cumsum(sizes)])
    rng = np.random.default_rng(2)
    w = rng.lognormal(size=len(src))
    g = K.Graph(int(off[-1]), src, tgt, w, False)
    try:
        K.set_tuning(K.TUNE_EGO_BIG_NODES, 50)
        K.set_tuning(K.TUNE_EGO_CLUSTER, cluster)
        out, its, info = g.pagerank_graphs(off, weighted=True, tol=1e-11)
        again, _, _ = g.pagerank_graphs(off, weighted=True, tol=1e-11)
        assert np.array_equal(out, again)
        assert info.hot_columns == cluster
        assert info.iterations_fp32 == int((sizes >= 50).sum()) > 0
        for k in range(len(sizes)):
            lo, hi = off[k], off[k + 1]
            sel = (src >= lo) & (src < hi)
            og = O.Graph(hi - lo, src[sel] - lo, tgt[sel] - lo, w[sel], False)
            ref = og.pagerank(weighted=True, tol=1e-11)
            assert np.abs(out[lo:hi] - ref).sum() <= 1e-12, k
            assert its[k] == og.last_iters, k
    finally:
        K.set_tuning(K.TUNE_EGO_BIG_NODES, 0)
        K.set_tuning(K.TUNE_EGO_CLUSTER, 0)


def test_pagerank_graphs_replays_its_launch_graph():
    """A repeated batch replays the instantiated launch graph (no new
    instantiation) with the same results; new teleport values are copied in
    and honoured without one; other parameters or another batch on the same
    handle instantiate again; every answer still matches the oracle."""
    sizes = np.array([40, 3, 120, 17, 64])
    src, tgt = K.generate_gnm(sizes, np.minimum(5 * sizes, sizes * (sizes - 1) // 2), False,
                              False, seed=31)
    off = np.concatenate([[0], np.cumsum(sizes)])
    g = K.Graph(int(off[-1]), src, tgt, None, False)

    def oracle(p=None, damping=0.85, offs=off):
        ref = np.zeros(int(offs[-1]))
        for k in range(len(offs) - 1):
            lo, hi = offs[k], offs[k + 1]
            sel = (src >= lo) & (src < hi)
            og = O.Graph(hi - lo, src[sel] - lo, tgt[sel] - lo, None, False)
            ref[lo:hi] = og.pagerank(personalization=None if p is None else p[lo:hi],
                                     damping=damping)
        return ref

    a, _, i1 = g.pagerank_graphs(off)
    b, _, i2 = g.pagerank_graphs(off)
    assert np.array_equal(a, b)
    assert i2.long_row == i1.long_row  # replayed, not instantiated again
    assert np.abs(a - oracle()).sum() <= 1e-12 * len(sizes)
    p = np.arange(off[-1], dtype=float) % 4 + 1
    c, _, i3 = g.pagerank_graphs(off, personalization=p)
    c2, _, i4 = g.pagerank_graphs(off, personalization=p[::-1].copy())
    assert i4.long_row == i3.long_row
    assert np.abs(c - oracle(p)).sum() <= 1e-12 * len(sizes)
    assert np.abs(c2 - oracle(p[::-1].copy())).sum() <= 1e-12 * len(sizes)
    d, _, i5 = g.pagerank_graphs(off, damping=0.6)
    assert i5.long_row == i4.long_row + 1
    assert np.abs(d - oracle(damping=0.6)).sum() <= 1e-12 * len(sizes)
    off2 = np.array([0, 43, off[-1]])  # graphs 0-1 and 2-4 taken together
    e, _, _ = g.pagerank_graphs(off2)
    assert np.abs(e - oracle(offs=off2)).sum() <= 1e-12 * 2


def test_pagerank_graphs_options_and_errors():
    sizes = np.array([7, 1, 30, 12])
    src, tgt = K.generate_gnm(sizes, np.minimum(2 * sizes, sizes * (sizes - 1) // 2), False,
                              False, seed=2)
    off = np.concatenate([[0], np.cumsum(sizes)])
    g = K.Graph(int(off[-1]), src, tgt, None, False)
    p = np.arange(off[-1], dtype=float) % 3 + 1
    out, _, _ = g.pagerank_graphs(off, personalization=p, dangling=1, loops=1, damping=0.7)
    for k in range(len(sizes)):
        lo, hi = off[k], off[k + 1]
        sel = (src >= lo) & (src < hi)
        og = O.Graph(hi - lo, src[sel] - lo, tgt[sel] - lo, None, False)
        ref = og.pagerank(personalization=p[lo:hi], dangling=1, loops=1, damping=0.7)
        assert np.abs(out[lo:hi] - ref).sum() <= 1e-12
    bad = K.Graph(10, [0, 3], [4, 9], None, False)
    with pytest.raises(K.EngineError, match="joins two different graphs"):
        bad.pagerank_graphs([0, 5, 10])
    with pytest.raises(K.EngineError, match="end at the node count"):
        g.pagerank_graphs([0, 5])
