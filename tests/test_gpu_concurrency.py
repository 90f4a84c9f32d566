"""Concurrent calls on shared handles. Handles are immutable and safe to read
from several threads at once (the reference's docs/EMBEDDING.md:24-29); the
library gives every calling thread its own stream and builds the cached
operators and workspaces under locks. Eight threads run PageRank (FP64 and
mixed), eigenvector centrality, Katz, HITS, components and degree on the
same handles, including a handle whose first call (which builds its
operators) happens in all threads at once; every result must be
bit-identical to the same call made alone.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import knappnet_b200 as K

pytestmark = pytest.mark.gpu


def calls(gd, gu):
    alpha = 0.5 / gd.eigenvector(mode=2, weighted=True)[1]
    return {
        "pagerank_fp64": lambda: gd.pagerank_ex(weighted=True, tol=1e-10,
                                                 precision=K.PREC_FP64)[0],
        "pagerank_mixed": lambda: gd.pagerank_ex(weighted=True, tol=1e-10,
                                                  precision=K.PREC_MIXED)[0],
        "pagerank_undirected": lambda: gu.pagerank(directed=False),
        "eigenvector": lambda: gu.eigenvector(mode=3)[0],
        "eigenvector_in": lambda: gd.eigenvector(mode=2, weighted=True)[0],
        "katz": lambda: gd.katz(alpha=alpha, mode=2, weighted=True),
        "hits": lambda: np.concatenate(gd.hits()[:2]),
        "strong": lambda: gd.components(strong=True)[0].astype(np.float64),
        "degree": lambda: gd.degree(mode=3, weighted=True),
    }


def graphs(seed):
    gd = K.generate_rmat(14, 16, seed=seed, clean=True, lognormal=True, wseed=seed + 1)
    gu = K.generate_rmat(14, 16, seed=seed + 2, clean=True, symmetrize=True)
    return gd, gu


def run_concurrently(fns, names, workers=8):
    with ThreadPoolExecutor(workers) as ex:
        futs = [(name, ex.submit(fns[name])) for name in names]
        return [(name, f.result()) for name, f in futs]


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


def test_concurrent_calls_match_serial_results():
    gd, gu = graphs(20241208)
    fns = calls(gd, gu)
    serial = {name: fn() for name, fn in fns.items()}
    names = [name for _ in range(4) for name in fns]
    for name, got in run_concurrently(fns, names):
        assert same(got, serial[name]), name
    gd.close()
    gu.close()


def test_first_use_from_many_threads():
    # the reference results come from an identical pair of handles
    ra, rb = graphs(20241210)
    serial = {name: fn() for name, fn in calls(ra, rb).items()}
    gd, gu = graphs(20241210)
    fns = calls(gd, gu)
    for name in ("pagerank_mixed", "eigenvector", "katz", "hits"):
        for got_name, got in run_concurrently(fns, [name] * 8):
            assert same(got, serial[got_name]), got_name
    for g in (ra, rb, gd, gu):
        g.close()
