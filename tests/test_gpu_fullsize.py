"""The benchmark configurations at their full sizes, through properties that
hold whatever the size (the CPU oracle is too slow to run the whole of them):

- directed weighted PageRank on R-MAT scale 24: the mixed path matches the
  all-FP64 path within 1e-9 L1 with the same top-100 order and the same
  stopping sweep, both sum to 1, and both are fixed points of the
  reference's update to within the stopping tolerance (checked on the host
  with an independent sparse product);
- eigenvector centrality by Lanczos on the symmetrised R-MAT scale 20 graph:
  the eigen-equation holds, and the FP64 and FP32-product variants agree;
- batched personalised PageRank on R-MAT scale 22 with 256 teleport
  vectors of 1-64 seed nodes each: every column sums to 1 and sampled
  columns match single-vector solves;
- 10,000 packed ego graphs (power-law sizes 50-50,000, mean degree 12):
  one launch, every graph sums to 1, sampled graphs match the oracle;
- differentiable PageRank on R-MAT scale 20: the adjoint gradient matches a
  central finite difference along a random direction on the whole graph,
  and per-edge central differences on the 1,000-node induced subgraph of
  the highest-degree nodes.
"""
from __future__ import annotations

import numpy as np
import pytest
import scipy.sparse as sp

import knappnet_b200 as K
from oracle import oracle as O

pytestmark = pytest.mark.gpu

D = 0.85


def pagerank_step(A, out_strength, x, d=D):
    """One reference update (spectral.rs:252-271) with uniform teleport:
    y = d (A_in (x / out) + stuck / n) + (1 - d) / n, normalised."""
    n = len(x)
    z = np.divide(x, out_strength, out=np.zeros_like(x), where=out_strength > 0)
    stuck = x[out_strength == 0].sum()
    y = d * (A @ z + stuck / n) + (1.0 - d) / n
    return y / y.sum()


def in_operator(g):
    off, cols, w = g.csr(1)
    n = g.n
    return sp.csr_matrix((w if w is not None else np.ones(len(cols)), cols.astype(np.int32),
                          off.astype(np.int64)), shape=(n, n))


def test_rmat24_mixed_matches_fp64_and_is_a_fixed_point():
    g = K.generate_rmat(24, 16, 0.57, 0.19, 0.19, seed=20240601, clean=True,
                        lognormal=True, wseed=20240602)
    x64, i64 = g.pagerank_ex(weighted=True, tol=1e-9, precision=K.PREC_FP64)
    xm, im = g.pagerank_ex(weighted=True, tol=1e-9, precision=K.PREC_MIXED)
    assert abs(x64.sum() - 1.0) < 1e-12 and abs(xm.sum() - 1.0) < 1e-12
    assert np.abs(xm - x64).sum() <= 1e-9
    assert im.iterations == i64.iterations
    top = np.argsort(-x64, kind="stable")[:100]
    assert np.array_equal(np.argsort(-xm, kind="stable")[:100], top)
    A = in_operator(g)
    outs = g.degree(mode=1, loops=True, weighted=True)
    for x in (x64, xm):
        assert np.abs(pagerank_step(A, outs, x) - x).sum() <= 1e-9
    g.close()


def test_rmat20_symmetric_lanczos_eigen_equation():
    g = K.generate_rmat(20, 16, seed=20240603, clean=True, symmetrize=True)
    x0, i0 = g.eigenvector_ex(mode=3, tol=1e-10, precision=0)
    x1, i1 = g.eigenvector_ex(mode=3, tol=1e-10, precision=1)
    off, cols, _ = g.csr(0)
    A = sp.csr_matrix((np.ones(len(cols)), cols.astype(np.int32), off.astype(np.int64)),
                      shape=(g.n, g.n))
    for x, info in ((x0, i0), (x1, i1)):
        lam = info.eigenvalue
        assert abs(x.max() - 1.0) < 1e-12
        assert np.abs(A @ x - lam * x).max() <= 1e-8 * lam
    assert abs(i0.eigenvalue - i1.eigenvalue) <= 1e-9 * i0.eigenvalue
    assert np.abs(x0 - x1).max() <= 1e-8
    g.close()


def test_rmat22_batch_256_vectors():
    g = K.generate_rmat(22, 16, seed=20240604, clean=True)
    n, B = g.n, 256
    rng = np.random.default_rng(20240605)
    P = np.zeros((B, n))
    for b in range(B):
        k = int(rng.integers(1, 65))
        P[b, rng.choice(n, size=k, replace=False)] = 1.0 / k
    out, info = g.pagerank_batch(P, precision=K.PREC_MIXED, tol=1e-10)
    assert np.abs(out.sum(axis=1) - 1.0).max() < 1e-12
    for b in (0, 1, 97, 255):
        ref, _ = g.pagerank_ex(personalization=P[b], tol=1e-10, precision=K.PREC_FP64)
        assert np.abs(out[b] - ref).sum() <= 1e-9, b
    assert info.max_column_iterations >= 1
    g.close()


def test_ten_thousand_ego_graphs_in_one_launch():
    sizes = K.power_law_sizes(10_000, 2.1, 50, 50_000, seed=20240606)
    m = np.minimum(6 * sizes, sizes * (sizes - 1) // 2)
    src, tgt = K.generate_gnm(sizes, m, False, False, seed=20240607)
    off = np.concatenate([[0], np.cumsum(sizes)])
    g = K.Graph(int(off[-1]), src, tgt, None, False)
    out, its, info = g.pagerank_graphs(off, tol=1e-12)
    assert info.kernel_launches == 1
    assert np.abs(np.add.reduceat(out, off[:-1]) - 1.0).max() < 1e-12
    rng = np.random.default_rng(3)
    picks = {int(np.argmax(sizes)), int(np.argmin(sizes))} | set(rng.choice(len(sizes), 10).tolist())
    for k in sorted(picks):
        lo, hi = off[k], off[k + 1]
        sel = (src >= lo) & (src < hi)
        og = O.Graph(hi - lo, src[sel] - lo, tgt[sel] - lo, None, False)
        ref = og.pagerank(tol=1e-12)
        # the oracle divides by a sequential sum; allow its own residual
        assert np.abs(out[lo:hi] - ref).sum() <= 1e-12 + abs(ref.sum() - 1.0), k
        assert its[k] == og.last_iters, k
    g.close()


def test_rmat20_adjoint_directional_and_subgraph_finite_differences():
    torch = pytest.importorskip("torch")
    from knappnet_b200 import autograd as AG
    g = K.generate_rmat(20, 16, seed=20240608, clean=True, lognormal=True, wseed=20240609)
    s, t, w = g.edges()
    rng = np.random.default_rng(20240610)
    pert = np.maximum(1 + 0.1 * rng.standard_normal(len(w)), 1e-3)

    def loss(wv, target):
        x = AG.pagerank(torch.tensor(wv, dtype=torch.float64, device="cuda"), g, tol=1e-13)
        return ((x - target) ** 2).sum().item()

    target = AG.pagerank(torch.tensor(w * pert, device="cuda"), g, tol=1e-13).detach()
    wt = torch.tensor(w, dtype=torch.float64, device="cuda", requires_grad=True)
    L = ((AG.pagerank(wt, g, tol=1e-13) - target) ** 2).sum()
    L.backward()
    grad = wt.grad.detach().cpu().numpy()
    v = rng.standard_normal(len(w)) * w
    h = 1e-4
    fd = (loss(w + h * v, target) - loss(w - h * v, target)) / (2 * h)
    an = float(grad @ v)
    assert abs(fd - an) <= 1e-5 * abs(an), (fd, an)

    # per-edge central differences on the 1,000-node induced subgraph of
    # the nodes of highest total degree
    deg = np.bincount(s, minlength=g.n) + np.bincount(t, minlength=g.n)
    keep = np.argsort(-deg, kind="stable")[:1000]
    idx = -np.ones(g.n, dtype=np.int64)
    idx[keep] = np.arange(1000)
    sel = (idx[s] >= 0) & (idx[t] >= 0)
    ss, tt, ws = idx[s[sel]], idx[t[sel]], w[sel]
    sg = K.Graph(1000, ss, tt, ws, True)
    tgt_s = AG.pagerank(torch.tensor(ws * pert[sel], device="cuda"), sg, tol=1e-15).detach()
    wst = torch.tensor(ws, dtype=torch.float64, device="cuda", requires_grad=True)
    ((AG.pagerank(wst, sg, tol=1e-15) - tgt_s) ** 2).sum().backward()
    gs = wst.grad.detach().cpu().numpy()

    def loss_s(wv):
        x = AG.pagerank(torch.tensor(wv, dtype=torch.float64, device="cuda"), sg, tol=1e-15)
        return ((x - tgt_s) ** 2).sum().item()

    for e in rng.choice(len(ws), 20, replace=False):
        he = 1e-4 * ws[e]
        wa, wb = ws.copy(), ws.copy()
        wa[e] += he
        wb[e] -= he
        fde = (loss_s(wa) - loss_s(wb)) / (2 * he)
        assert abs(fde - gs[e]) <= 1e-5 * max(abs(fde), 1e-3 * np.abs(gs).max()), (e, fde, gs[e])
    sg.close()
    g.close()
