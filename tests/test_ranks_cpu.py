"""The multi-process plumbing on CPU: two gloo ranks, as torchrun would
start them, reduce the benchmark's timing (maximum over ranks) and units
(sum over ranks), and the no-exchange splits of teleport vectors and packed
graphs partition the work exactly."""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from knappnet_b200 import ranks


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, queue):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    r, w, _, dist = ranks.init("gloo", timeout_s=60.0)
    ranks.barrier(dist)
    t = ranks.max_over_ranks(dist, 1.5 + r)     # per-rank device seconds
    u = ranks.sum_over_ranks(dist, 1000.0 * (r + 1))  # per-rank arcs x sweeps
    lo, hi = ranks.split_columns(256, w, r)
    cols = ranks.sum_over_ranks(dist, hi - lo)
    queue.put((r, w, t, u, lo, hi, cols))
    dist.destroy_process_group()


def test_two_gloo_ranks_reduce_and_split():
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    assert all(r[2] == 2.5 for r in res)      # the slowest rank's time
    assert all(r[3] == 3000.0 for r in res)   # units of the whole job
    assert (res[0][4], res[0][5], res[1][4], res[1][5]) == (0, 128, 128, 256)
    assert all(r[6] == 256 for r in res)


def _gather_worker(rank, world, port, queue):
    import torch
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    r, w, _, dist = ranks.init("gloo", timeout_s=60.0)
    # 7 teleport vectors of 5 scores: rank r holds its column range
    ranges = [ranks.split_columns(7, w, k) for k in range(w)]
    lo, hi = ranges[r]
    full = np.arange(35, dtype=np.float64).reshape(7, 5)
    got = ranks.gather_rows(dist, torch.from_numpy(full[lo:hi].copy()), ranges)
    # packed graphs: per-node scores of the graphs each rank solved
    sizes = np.array([3, 1, 4, 1, 5, 9, 2, 6])
    off = np.concatenate([[0], np.cumsum(sizes)])
    cuts = [ranks.split_graphs(off, 2 * sizes, w, k) for k in range(w)]
    nodes = [(int(off[a]), int(off[b])) for a, b in cuts]
    a, b = nodes[r]
    scores = np.linspace(0.0, 1.0, int(off[-1]))
    got2 = ranks.gather_rows(dist, torch.from_numpy(scores[a:b].copy()), nodes)
    queue.put((r, None if got is None else got.tolist(), None if got2 is None else got2.tolist()))
    dist.destroy_process_group()


def test_two_gloo_ranks_gather_their_parts_in_order():
    """Rank 0 reassembles teleport columns and packed-graph scores in the
    original order from parts of different lengths; the other rank gets
    nothing back."""
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((x for x in (q.get(timeout=120) for _ in procs)), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    full = np.arange(35, dtype=np.float64).reshape(7, 5)
    assert np.array_equal(np.array(res[0][1]), full)
    assert np.array_equal(np.array(res[0][2]), np.linspace(0.0, 1.0, 31))
    assert res[1][1] is None and res[1][2] is None


def test_single_process_reductions_are_identities():
    assert ranks.max_over_ranks(None, 3.0) == 3.0
    assert ranks.sum_over_ranks(None, 3.0) == 3.0
    ranks.barrier(None)


@pytest.mark.parametrize("batch,world", [(256, 1), (256, 3), (10, 4), (3, 8), (0, 2)])
def test_split_columns_partitions(batch, world):
    got = [ranks.split_columns(batch, world, r) for r in range(world)]
    assert got[0][0] == 0 and got[-1][1] == batch
    assert all(got[k][1] == got[k + 1][0] for k in range(world - 1))
    sizes = [hi - lo for lo, hi in got]
    assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_split_graphs_partitions_and_balances(world):
    rng = np.random.default_rng(world)
    sizes = np.maximum(rng.pareto(1.1, 10_000) * 50, 50).astype(np.int64).clip(50, 50_000)
    arcs = 12 * sizes
    off = np.concatenate([[0], np.cumsum(sizes)])
    cuts = [ranks.split_graphs(off, arcs, world, r) for r in range(world)]
    assert cuts[0][0] == 0 and cuts[-1][1] == len(sizes)
    assert all(cuts[k][1] == cuts[k + 1][0] for k in range(world - 1))
    work = sizes + arcs
    share = np.array([work[a:b].sum() for a, b in cuts]) / work.sum()
    assert np.abs(share - 1.0 / world).max() <= work.max() / work.sum() + 1e-12


def test_split_rejects_bad_ranks():
    with pytest.raises(ValueError):
        ranks.split_columns(10, 2, 2)
    with pytest.raises(ValueError):
        ranks.split_graphs([0, 5], [3], 0, 0)
