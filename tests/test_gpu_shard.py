"""Row shards of one graph's PageRank on a B200, through the C ABI
(net_shard_*). The ranks of a split solve run in one process, one after
another: each rank's sweep writes its slice of one buffer laid out as the
all-gather leaves it, then every rank finishes the sweep from that buffer.
No kernel waits on another. Every rank must hold the same iterate bit for
bit, and the scores and sweep count must be the oracle's
(crates/engine/src/metrics/spectral.rs:247-280) and net_pagerank's, in node
order (shards work on the rows renumbered by column count). A group of one
runs ranks.pagerank_rows over NCCL in a child process."""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import numpy as np
import pytest

import knappnet_b200 as K
from oracle import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def split_solve(g, parts, tol=1e-12, max_iter=10000, pers=None, **opts):
    """The split solve with `parts` ranks emulated in turn; returns the
    scores, the sweeps and the boundaries."""
    import torch
    b = g.shard_bounds(parts, directed=opts.get("directed", True),
                       weighted=opts.get("weighted", False), loops=opts.get("loops", 0))
    pp = None
    if pers is not None:
        pt = torch.tensor(pers, dtype=torch.float64, device="cuda")
        pp = pt.data_ptr()
    shards = [K.Shard(g, b, r, personalization_ptr=pp, **opts) for r in range(parts)]
    L = shards[0].payload_len
    assert all(s.payload_len == L for s in shards)
    buf = torch.empty(parts * L, dtype=torch.float64, device="cuda")
    sweeps = 0
    for sweeps in range(1, max_iter + 1):
        for r, s in enumerate(shards):
            s.sweep(buf[r * L:(r + 1) * L])
        changes = [s.finish(buf) for s in shards]
        assert len(set(changes)) == 1
        if changes[0] <= tol:
            break
    xs = [s.scores() for s in shards]
    for x in xs[1:]:
        assert np.array_equal(x, xs[0])
    for s in shards:
        s.close()
    return xs[0], sweeps, b


def random_graph(seed, n, m, loops=True, dangling=True):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, n, m)
    tgt = rng.integers(0, n, m)
    if not loops:
        keep = src != tgt
        src, tgt = src[keep], tgt[keep]
    if dangling:  # the last tenth of the nodes sends nothing
        src = np.where(src >= n - n // 10, src % (n - n // 10), src)
    w = rng.random(len(src)) * 3 + 0.01
    return n, src, tgt, w


CASES = [
    dict(directed=True, weighted=True, loops=0),
    dict(directed=True, weighted=False, loops=2),
    dict(directed=False, weighted=True, loops=1),
    dict(directed=False, weighted=False, loops=0),
]


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_split_pagerank_matches_oracle(parts, case):
    opts = CASES[case]
    for directed_graph in (True, False):
        n, src, tgt, w = random_graph(100 + case, 700, 4000)
        g = K.Graph(n, src, tgt, w, directed_graph)
        og = O.Graph(n, src, tgt, w, directed_graph)
        x, sweeps, b = split_solve(g, parts, **opts)
        ref = og.pagerank(tol=1e-12, **opts)
        assert np.abs(x - ref).sum() <= 1e-12, (opts, directed_graph)
        assert sweeps == og.last_iters
        single, info = g.pagerank_ex(tol=1e-12, **opts)
        assert np.abs(x - single).sum() <= 1e-12
        assert b[0] == 0 and b[-1] == n and np.all(np.diff(b) >= 0)


@pytest.mark.parametrize("dangling", [0, 1])
def test_split_pagerank_with_personalization(dangling):
    n, src, tgt, w = random_graph(7, 500, 3000)
    g = K.Graph(n, src, tgt, w, True)
    og = O.Graph(n, src, tgt, w, True)
    p = np.random.default_rng(8).random(n) * 5  # rescaled to sum 1 by the shard
    p[::7] = 0.0
    x, sweeps, _ = split_solve(g, 3, pers=p, dangling=dangling, weighted=True)
    ref = og.pagerank(weighted=True, personalization=p, dangling=dangling, tol=1e-12)
    assert np.abs(x - ref).sum() <= 1e-12
    assert sweeps == og.last_iters


def test_split_pagerank_rmat_against_single_gpu_and_oracle():
    g = K.generate_rmat(14, 16, seed=21, clean=True, lognormal=True, wseed=22)
    s, t, w = g.edges()
    og = O.Graph(g.n, s, t, w, True)
    x, sweeps, b = split_solve(g, 4, weighted=True)
    ref = og.pagerank(weighted=True, tol=1e-12)
    assert np.abs(x - ref).sum() <= 1e-12 and sweeps == og.last_iters
    single, info = g.pagerank_ex(weighted=True, tol=1e-12)
    assert np.abs(x - single).sum() <= 1e-12 and info.iterations == sweeps
    # ranges over the rows renumbered by column count, each holding rows
    assert b[0] == 0 and b[-1] == g.n and np.all(np.diff(b) > 0)


def test_more_ranks_than_rows_and_the_empty_graph():
    n, src, tgt, w = random_graph(3, 5, 9, dangling=False)
    g = K.Graph(n, src, tgt, w, True)
    og = O.Graph(n, src, tgt, w, True)
    x, sweeps, b = split_solve(g, 8, weighted=True)
    assert (np.diff(b) == 0).any()  # some ranks hold no rows
    ref = og.pagerank(weighted=True, tol=1e-12)
    assert np.abs(x - ref).sum() <= 1e-12 and sweeps == og.last_iters
    import torch
    from knappnet_b200 import ranks
    e = K.Graph(0, [], [], None, True)
    sh = K.Shard(e, e.shard_bounds(2), 1)
    assert ranks.pagerank_rows(None, sh, device="cuda") == 0
    assert sh.scores().shape == (0,)


def test_restart_returns_to_the_uniform_iterate():
    n, src, tgt, w = random_graph(4, 300, 2000)
    g = K.Graph(n, src, tgt, w, True)
    from knappnet_b200 import ranks
    sh = K.Shard(g, g.shard_bounds(1), 0)
    assert np.all(sh.scores() == 1.0 / n)
    s1 = ranks.pagerank_rows(None, sh, device="cuda", tol=1e-12)
    x1 = sh.scores()
    sh.restart()
    assert np.all(sh.scores() == 1.0 / n)
    s2 = ranks.pagerank_rows(None, sh, device="cuda", tol=1e-12)
    assert s1 == s2 and np.array_equal(sh.scores(), x1)
    with pytest.raises(K.EngineError, match="did not converge to tolerance 0.000000 within 2"):
        sh.restart()
        ranks.pagerank_rows(None, sh, device="cuda", tol=1e-12, max_iter=2)


def test_shard_errors_name_the_problem():
    n, src, tgt, w = random_graph(5, 50, 200)
    g = K.Graph(n, src, tgt, w, True)
    b = g.shard_bounds(2)
    with pytest.raises(K.EngineError, match="must not decrease"):
        K.Shard(g, [0, 30, 20, n], 0)
    with pytest.raises(K.EngineError, match="end at the node count 50"):
        K.Shard(g, [0, 20, 49], 0)
    with pytest.raises(K.EngineError, match=r"shard 2 is outside \[0, 2\)"):
        K.Shard(g, b, 2)
    with pytest.raises(K.EngineError, match="between 1 and 1024"):
        g.shard_bounds(0)
    with pytest.raises(K.EngineError, match="between 1 and 1024"):
        g.shard_bounds(1025)
    with pytest.raises(K.EngineError, match="unknown dangling-node code 2"):
        K.Shard(g, b, 0, dangling=2)
    with pytest.raises(K.EngineError, match="unknown self-loop weight code 3"):
        K.Shard(g, b, 0, loops=3)
    with pytest.raises(K.EngineError, match="damping is 1.5; it must be between 0 and 1"):
        K.Shard(g, b, 0, damping=1.5)
    neg = K.Graph(3, [0, 1], [1, 2], [1.0, -2.0], True)
    with pytest.raises(K.EngineError, match="negative weight"):
        K.Shard(neg, neg.shard_bounds(1), 0, weighted=True)
    import torch
    bad = torch.tensor([1.0, -1.0] + [1.0] * (n - 2), dtype=torch.float64, device="cuda")
    with pytest.raises(K.EngineError, match="finite, nonnegative"):
        K.Shard(g, b, 0, personalization_ptr=bad.data_ptr())


NCCL_CHILD = r"""
import numpy as np, torch, knappnet_b200 as K
from knappnet_b200 import ranks
r, w, local, dist = ranks.init("nccl", timeout_s=60.0)
g = K.generate_rmat(12, 16, seed=3, clean=True, lognormal=True, wseed=4)
sh = K.Shard(g, g.shard_bounds(w, directed=True, weighted=True), r, weighted=True)
sweeps = ranks.pagerank_rows(dist, sh, device=torch.device("cuda", local), tol=1e-12)
ref, info = g.pagerank_ex(weighted=True, tol=1e-12)
print("RESULT", sweeps, info.iterations, float(np.abs(sh.scores() - ref).sum()), flush=True)
sh.close()
dist.destroy_process_group()
"""


def test_group_of_one_exchanges_over_nccl():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0", MASTER_ADDR="127.0.0.1",
               MASTER_PORT=str(port), NCCL_NVLS_ENABLE="0")
    r = subprocess.run([sys.executable, "-c", NCCL_CHILD], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("RESULT")][0].split()
    sweeps, iters, l1 = int(line[1]), int(line[2]), float(line[3])
    assert sweeps == iters and l1 <= 1e-12
