"""One process per GPU: rank set-up, reductions over ranks, the splits of
the workloads that shard with no exchange, and the row split of one graph's
PageRank.

The batched and packed-graph workloads split with no exchange at all:
teleport vectors by contiguous column ranges, packed graphs by contiguous
graph ranges balanced by their nodes plus arcs; each rank solves its part
alone, and the parts are assembled on rank 0 afterwards (gather_rows).
PageRank on one graph splits by rows of its pull operator with one exchange
per sweep (pagerank_rows): every rank sweeps its rows, the ranks all-gather
their payloads, and every rank finishes the sweep over all nodes. Reductions
and gathers run on the process group's own device (CUDA tensors for NCCL,
CPU tensors for gloo), so the same code serves the GPU runs and the CPU
tests.
"""
from __future__ import annotations

import os
from datetime import timedelta

import numpy as np


def rank_env():
    """(rank, world, local rank) from the torchrun environment (0, 1, 0
    when launched as a single process)."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def init(backend: str = "nccl", timeout_s: float = 300.0):
    """Joins the process group of a torchrun launch; returns (rank, world,
    local, dist) with dist None for a single process."""
    rank, world, local = rank_env()
    if world <= 1 and "WORLD_SIZE" not in os.environ:
        return 0, 1, 0, None
    import torch
    import torch.distributed as dist
    kw = {}
    if backend == "nccl":
        torch.cuda.set_device(local)
        kw["device_id"] = torch.device("cuda", local)
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s), **kw)
    return rank, world, local, dist


def _reduce(dist, x: float, op) -> float:
    if dist is None:
        return float(x)
    import torch
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(dist, x: float) -> float:
    """The largest x over all ranks (device time of the slowest rank)."""
    return _reduce(dist, x, None if dist is None else dist.ReduceOp.MAX)


def sum_over_ranks(dist, x: float) -> float:
    """The sum of x over all ranks (units processed by the whole job)."""
    return _reduce(dist, x, None if dist is None else dist.ReduceOp.SUM)


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def split_columns(batch: int, world: int, rank: int):
    """The contiguous range [lo, hi) of teleport vectors this rank solves:
    sizes differ by at most one and the ranges cover 0..batch exactly."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in 0..world-1")
    q, r = divmod(int(batch), world)
    lo = rank * q + min(rank, r)
    return lo, lo + q + (1 if rank < r else 0)


def split_graphs(node_offsets, arc_counts, world: int, rank: int):
    """The contiguous range [g0, g1) of packed graphs this rank solves, cut
    where the running work (nodes plus arcs per graph) crosses rank/world of
    the total, so ranks get nearly equal work; the ranges cover all graphs
    exactly once, in order."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must lie in 0..world-1")
    off = np.asarray(node_offsets, dtype=np.int64)
    work = np.diff(off) + np.asarray(arc_counts, dtype=np.int64)
    cum = np.concatenate([[0], np.cumsum(work)])
    total = cum[-1]
    cuts = [int(np.searchsorted(cum, total * k / world, side="left")) for k in range(world + 1)]
    cuts[0], cuts[-1] = 0, len(work)
    for k in range(1, world + 1):
        cuts[k] = max(cuts[k], cuts[k - 1])
    return cuts[rank], cuts[rank + 1]


def gather_rows(dist, local, ranges):
    """Assembles on rank 0 the rows every rank computed: rank r holds rows
    ranges[r] = (lo, hi) of a result whose rows follow the ranges in rank
    order, as `local` (a tensor of shape (hi - lo, ...) on the group's
    device). Parts are padded to the longest for the collective and cut
    back. Returns the whole result as a numpy array on rank 0 and None on
    the other ranks (the local part itself, as numpy, for a single
    process)."""
    if dist is None:
        return local.cpu().numpy()
    import torch
    world = dist.get_world_size()
    if len(ranges) != world:
        raise ValueError("one row range per rank")
    longest = max(hi - lo for lo, hi in ranges)
    shape = (longest,) + tuple(local.shape[1:])
    pad = torch.zeros(shape, dtype=local.dtype, device=local.device)
    pad[: local.shape[0]] = local
    parts = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad)
    if dist.get_rank() != 0:
        return None
    return torch.cat([parts[r][: hi - lo] for r, (lo, hi) in enumerate(ranges)]).cpu().numpy()


def all_gather_flat(dist, out, local) -> None:
    """out (world * len(local) values) <- every rank's `local`, in rank
    order: one all_gather_into_tensor where the backend has it (NCCL), else
    the list form."""
    world = dist.get_world_size()
    if dist.get_backend() == "nccl":
        dist.all_gather_into_tensor(out, local)
        return
    parts = list(out.view(world, -1).unbind(0))
    dist.all_gather(parts, local)


def pagerank_rows(dist, shard, device=None, tol=0.0, max_iter=0):
    """PageRank of one graph split over the ranks by rows; returns the number
    of sweeps (the scores stay in the shard). `shard` is this rank's row
    shard (knappnet_b200.Shard): a sweep writes its payload_len-value
    payload, the ranks all-gather the payloads (one collective per sweep,
    also for a group of one; none without a group, `dist` None), and the
    shard finishes the sweep over all nodes from them, returning the L1
    change. Every rank
    computes the same change, so all ranks stop on the same sweep, at the
    first change <= tol, as net_pagerank (a tolerance that is not positive
    selects 1e-12, an iteration cap that is not positive 10000); at the cap
    it raises EngineError with net_pagerank's message."""
    import torch
    from . import EngineError
    tol = tol if tol > 0 else 1e-12
    max_iter = int(max_iter) if max_iter > 0 else 10000
    if shard.n == 0:
        return 0
    world = dist.get_world_size() if dist is not None else 1
    L = shard.payload_len
    send = torch.empty(L, dtype=torch.float64, device=device)
    recv = send if dist is None else torch.empty(world * L, dtype=torch.float64, device=device)
    for sweep in range(1, max_iter + 1):
        shard.sweep(send)
        if dist is not None:
            all_gather_flat(dist, recv, send)
        if shard.finish(recv) <= tol:
            return sweep
    raise EngineError(f"PageRank did not converge to tolerance {tol:f} within {max_iter} "
                      "iterations")
