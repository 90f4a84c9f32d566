"""Differentiable PageRank: the hand-written adjoint against dense torch
autograd (FP64) and central finite differences."""
from __future__ import annotations

import numpy as np
import pytest

import knappnet_b200 as K

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def dense_pagerank(w, src, tgt, n, d, directed, loops_factor=1.0):
    """PageRank by a dense solve: M[i, j] = sum of w over arcs j -> i / s_j,
    x = solve(I - d M - d jump 1_D^T, (1 - d) p), uniform p and jump."""
    A = torch.zeros((n, n), dtype=torch.float64, device=w.device)
    s_ = torch.as_tensor(src, device=w.device)
    t_ = torch.as_tensor(tgt, device=w.device)
    f = torch.where(s_ == t_, torch.as_tensor(loops_factor, dtype=torch.float64, device=w.device),
                    torch.ones((), dtype=torch.float64, device=w.device))
    A = A.index_put((t_, s_), w * f, accumulate=True)
    if not directed:
        off = s_ != t_
        A = A.index_put((s_[off], t_[off]), w[off], accumulate=True)
    out = A.sum(dim=0)
    dang = out == 0
    M = A / torch.where(dang, torch.ones_like(out), out)
    jump = torch.full((n,), 1.0 / n, dtype=torch.float64, device=w.device)
    G = M + torch.outer(jump, dang.to(torch.float64))
    I = torch.eye(n, dtype=torch.float64, device=w.device)
    x = torch.linalg.solve(I - d * G, (1 - d) * jump)
    return x / x.sum()


def random_weighted(n, m, seed, directed=True):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, n, m)
    tgt = rng.integers(0, n, m)
    # some dangling nodes: no arcs out of the last tenth
    src = np.where(src >= n - n // 10, src - n // 10, src)
    w = rng.lognormal(size=m)
    return src, tgt, w


@pytest.mark.parametrize("directed", [True, False])
def test_adjoint_matches_dense_autograd(directed):
    from knappnet_b200 import autograd as A
    n, m = 300, 2400
    src, tgt, w = random_weighted(n, m, 3, directed)
    g = K.Graph(n, src, tgt, w, directed)
    wt = torch.tensor(w, dtype=torch.float64, device="cuda", requires_grad=True)
    target = torch.rand(n, dtype=torch.float64, device="cuda") / n
    x = A.pagerank(wt, g, tol=1e-14)
    loss = ((x - target) ** 2).sum()
    loss.backward()
    ours = wt.grad.detach().clone()
    wd = torch.tensor(w, dtype=torch.float64, device="cuda", requires_grad=True)
    xd = dense_pagerank(wd, src, tgt, n, 0.85, directed, 1.0 if directed else 2.0)
    assert torch.abs(x.detach() - xd.detach()).sum().item() <= 1e-12
    ld = ((xd - target) ** 2).sum()
    ld.backward()
    ref = wd.grad.detach()
    err = torch.abs(ours - ref).max().item()
    scale = torch.abs(ref).max().item()
    assert err <= 1e-9 * scale, (err, scale)


def test_adjoint_finite_differences_on_rmat_subgraph():
    from knappnet_b200 import autograd as A
    # 1,000-node induced subgraph of an R-MAT graph: the 1,000 nodes of
    # highest total degree
    big = K.generate_rmat(12, 16, seed=4, clean=True, lognormal=True, wseed=5)
    s, t, w = big.edges()
    deg = np.bincount(s, minlength=big.n) + np.bincount(t, minlength=big.n)
    keep = np.argsort(-deg, kind="stable")[:1000]
    idx = -np.ones(big.n, dtype=np.int64)
    idx[keep] = np.arange(1000)
    sel = (idx[s] >= 0) & (idx[t] >= 0)
    src, tgt, w = idx[s[sel]], idx[t[sel]], w[sel]
    g = K.Graph(1000, src, tgt, w, True)
    rng = np.random.default_rng(7)
    wt = torch.tensor(w, dtype=torch.float64, device="cuda", requires_grad=True)
    # target: PageRank with weights perturbed by 10%
    wp = torch.tensor(w * np.maximum(1 + 0.1 * rng.standard_normal(len(w)), 1e-3),
                      dtype=torch.float64, device="cuda")
    target = A.pagerank(wp, g, tol=1e-15).detach()
    x = A.pagerank(wt, g, tol=1e-15)
    loss = ((x - target) ** 2).sum()
    loss.backward()
    grad = wt.grad.detach().cpu().numpy()
    picks = rng.choice(len(w), 25, replace=False)
    for e in picks:
        h = 1e-4 * w[e]
        wa = w.copy()
        wa[e] += h
        wb = w.copy()
        wb[e] -= h
        la = ((A.pagerank(torch.tensor(wa, device="cuda"), g, tol=1e-15) - target) ** 2).sum()
        lb = ((A.pagerank(torch.tensor(wb, device="cuda"), g, tol=1e-15) - target) ** 2).sum()
        fd = (la - lb).item() / (2 * h)
        assert abs(fd - grad[e]) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(grad).max()), (e, fd, grad[e])


def test_weights_forward_matches_graph_weights():
    kg = K.generate_rmat(11, 16, seed=8, clean=True, lognormal=True, wseed=9)
    _, _, w = kg.edges()
    a = kg.pagerank(weighted=True)
    out = torch.empty(kg.n, dtype=torch.float64, device="cuda")
    wt = torch.tensor(w, device="cuda")
    import ctypes
    info = K.NetSolveInfo()
    err = ctypes.create_string_buffer(K.ERR_LEN)
    K._check(K.lib().net_pagerank_weights_device(kg.h, ctypes.c_void_p(wt.data_ptr()), 0.85, 1,
                                                 None, 0, 0, 0.0, 0, 0,
                                                 ctypes.c_void_p(out.data_ptr()),
                                                 ctypes.byref(info), err, K.ERR_LEN), err)
    assert np.abs(out.cpu().numpy() - a).sum() <= 1e-12
