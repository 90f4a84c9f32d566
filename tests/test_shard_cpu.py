"""The row split of one graph's PageRank on CPU: two and three gloo ranks run
ranks.pagerank_rows, the driver every GPU rank runs, with a numpy shard that
keeps the C ABI's payload contract (net_shard_sweep / net_shard_finish: the
rank's unnormalised rows, zero padding, its partial sum in the last slot;
the finish over all nodes from the payloads gathered in rank order). All
ranks must end with the same scores on the same sweep, and those must be
the oracle's PageRank (crates/engine/src/metrics/spectral.rs:247-280)."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from knappnet_b200 import ranks
from oracle import oracle as O


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _graph(seed=5, n=300, m=1500):
    rng = np.random.default_rng(seed)
    src = rng.integers(0, n, m)
    tgt = rng.integers(0, n, m)
    keep = src != tgt  # no self-loops: their diagonal factor is not restated here
    src, tgt = src[keep], tgt[keep]
    src[:5] = tgt[:5] = 0  # node 0 gets no out-arcs from these: dangling nodes exist
    keep = src != tgt
    w = rng.random(len(src))[keep] + 0.1
    return n, src[keep], tgt[keep], w


def _bounds(n, src, tgt, parts):
    """Row boundaries balancing rows plus in-arcs, as net_shard_bounds."""
    indeg = np.bincount(tgt, minlength=n)
    off = np.concatenate([[0], np.cumsum(indeg)])
    f = np.arange(n + 1) + off
    total = n + len(src)
    return np.array([int(np.searchsorted(f, total * k // parts, side="left"))
                     for k in range(parts + 1)], dtype=np.int64)


class NumpyShard:
    """Rows [b[rank], b[rank + 1]) of the pull operator of a directed,
    weighted graph without self-loops, uniform teleport."""

    def __init__(self, n, src, tgt, w, bounds, rank, damping=0.85):
        self.n, self.d = n, damping
        self.b = [int(v) for v in bounds]
        self.parts = len(self.b) - 1
        self.r0, self.r1 = self.b[rank], self.b[rank + 1]
        widest = max(self.b[k + 1] - self.b[k] for k in range(self.parts))
        self.payload_len = (widest + 1 + 31) // 32 * 32
        self.A = np.zeros((n, n))
        np.add.at(self.A, (tgt, src), w)
        self.out = self.A.sum(axis=0)
        self.x = np.full(n, 1.0 / n)
        self._prepare()

    def _prepare(self):
        dang = self.out <= 0
        self.z = np.where(dang, 0.0, self.x / np.where(dang, 1.0, self.out))
        self.stuck = float(self.x[dang].sum())

    def sweep(self, payload):
        import torch
        y = self.A[self.r0:self.r1] @ self.z
        y = self.d * (y + self.stuck / self.n) + (1.0 - self.d) / self.n
        buf = np.zeros(self.payload_len)
        buf[: len(y)] = y
        buf[-1] = y.sum()
        payload.copy_(torch.from_numpy(buf))

    def finish(self, gathered) -> float:
        g = gathered.numpy().reshape(self.parts, self.payload_len)
        total = sum(g[k, -1] for k in range(self.parts))
        y = np.concatenate([g[k, : self.b[k + 1] - self.b[k]] for k in range(self.parts)])
        xn = y / total
        change = float(np.abs(xn - self.x).sum())
        self.x = xn
        self._prepare()
        return change


def _worker(rank, world, port, queue):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    r, w, _, dist = ranks.init("gloo", timeout_s=60.0)
    n, src, tgt, wt = _graph()
    sh = NumpyShard(n, src, tgt, wt, _bounds(n, src, tgt, w), r)
    sweeps = ranks.pagerank_rows(dist, sh, device="cpu", tol=1e-12)
    queue.put((r, sweeps, sh.x.tolist()))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_split_pagerank_by_rows(world):
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    s0, x0 = res[0][1], res[0][2]
    for _, s, x in res[1:]:
        assert s == s0 and x == x0  # the same stopping sweep and iterate on every rank
    n, src, tgt, w = _graph()
    og = O.Graph(n, src, tgt, w, True)
    ref = og.pagerank(directed=True, weighted=True, tol=1e-12)
    assert np.abs(np.array(x0) - ref).sum() <= 1e-12
    assert s0 == og.last_iters


def test_single_process_row_split_and_the_iteration_cap():
    pytest.importorskip("torch")
    n, src, tgt, w = _graph(seed=9)
    sh = NumpyShard(n, src, tgt, w, _bounds(n, src, tgt, 1), 0)
    sweeps = ranks.pagerank_rows(None, sh, device="cpu", tol=1e-12)
    og = O.Graph(n, src, tgt, w, True)
    ref = og.pagerank(directed=True, weighted=True, tol=1e-12)
    assert np.abs(sh.x - ref).sum() <= 1e-12 and sweeps == og.last_iters
    from knappnet_b200 import EngineError
    sh = NumpyShard(n, src, tgt, w, _bounds(n, src, tgt, 1), 0)
    with pytest.raises(EngineError, match="did not converge to tolerance 0.000000 within 3"):
        ranks.pagerank_rows(None, sh, device="cpu", tol=1e-12, max_iter=3)


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_bounds_balance_rows_plus_arcs(parts):
    n, src, tgt, _ = _graph()
    b = _bounds(n, src, tgt, parts)
    assert b[0] == 0 and b[-1] == n and np.all(np.diff(b) >= 0)
    indeg = np.bincount(tgt, minlength=n)
    load = [int(b[k + 1] - b[k] + indeg[b[k]:b[k + 1]].sum()) for k in range(parts)]
    assert max(load) - min(load) <= 2 * (indeg.max() + 1)


def test_shard_buffers_are_checked_before_any_device_call():
    torch = pytest.importorskip("torch")
    import knappnet_b200 as K
    with pytest.raises(ValueError, match="contiguous float64 CUDA tensor"):
        K._dev_ptr(torch.zeros(4, dtype=torch.float64), 4)
    with pytest.raises(ValueError, match="contiguous float64 CUDA tensor"):
        K._dev_ptr(torch.zeros(4, dtype=torch.float32), 4)
    assert K._dev_ptr(1 << 20).value == 1 << 20  # a raw device address passes through
