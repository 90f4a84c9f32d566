"""Reads the packed golden file and runs a manifest variant on an engine.

An "engine" is any object with the reference's graph and measure calls
(oracle.oracle.Graph, or knappnet_b200.Graph over the CUDA library), so the
same variant code checks the oracle and the product.
"""
from __future__ import annotations

import json
import math
from functools import lru_cache
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "spectral_golden.json"

MODES = {"out": 1, "in": 2, "all": 3}
LOOPS = {"twice": 0, "once": 1, "ignore": 2}
DANGLING = {"personalized": 0, "uniform": 1}
SCALES = {"max": 0, "unit": 1}
HITS_SCALES = {"max": 0, "sum": 1, "unit": 2}


@lru_cache(maxsize=1)
def load():
    return json.loads(GOLDEN.read_text())


def node_rule(rule: str, n: int):
    """validation/bindings/spectral.py:84-96 (the rules on this path)."""
    if rule == "mod3plus1":
        return [float(v % 3 + 1) for v in range(n)]
    raise ValueError(rule)


def applies(spec: dict, fx: dict) -> bool:
    kind = spec.get("applies_to", "any")
    if kind == "directed" and not fx["directed"]:
        return False
    if kind == "undirected" and fx["directed"]:
        return False
    if spec.get("requires_weights") and not fx["weighted"]:
        return False
    return True


def cases():
    """(fixture, variant, oracle) triples that have a golden vector."""
    doc = load()
    out = []
    for fx_name, per in doc["golden"].items():
        fx = doc["fixtures"][fx_name]
        for variant, oracles in per.items():
            if not applies(doc["manifest"][variant], fx):
                continue
            for oracle in oracles:
                out.append((fx_name, variant, oracle))
    return out


def make_graph(graph_cls, fx: dict):
    w = None if fx["w"] is None else np.asarray(fx["w"], dtype=np.float64)
    return graph_cls(fx["n"], np.asarray(fx["src"], dtype=np.int64),
                     np.asarray(fx["tgt"], dtype=np.int64), w, fx["directed"])


def spectral_radius(g, mode: str, weighted: bool, loops: str) -> float:
    """Largest eigenvalue of the matrix a measure uses, from the engine's own
    eigenvector centrality (validation/bindings/spectral.py:140-151)."""
    _, lam, _ = g.eigenvector(mode=MODES[mode], weighted=weighted, scale=0, loops=LOOPS[loops])
    return lam


def relative(e: dict, key: str, g, mode: str, weighted: bool, loops: str) -> float:
    """`key` as given, or `key_fraction` / lambda_max
    (validation/bindings/spectral.py:154-161)."""
    if key in e:
        return float(e[key])
    lam = spectral_radius(g, mode, weighted, loops)
    if lam <= 0.0:
        return float(e[key + "_fraction"])
    return float(e[key + "_fraction"]) / lam


def target(g, e: dict):
    """The graph, or its adjacency-matrix reading (net_graph_simplify) when
    the variant says `simple` or `symmetrize`
    (validation/bindings/topography.py:64-85,157; spectral.py:118-137)."""
    if e.get("symmetrize"):
        return g.simplify(undirected=True, keep=0)
    if e.get("simple"):
        return g.simplify(undirected=False, keep=0)
    return g


def defined(values):
    """NaN written as -1, as the topography and two-mode runners do
    (validation/bindings/topography.py:17,60-61)."""
    return [-1.0 if math.isnan(v) else float(v) for v in values]


def run_variant(g, fx: dict, variant: str):
    """Runs the manifest's engine options for `variant` on graph `g`; a
    measure the engine rejects gives an empty vector, as in the reference's
    harness (validation/bindings/spectral.py:163-169)."""
    try:
        return _run_variant(g, fx, variant)
    except RuntimeError:  # the engines' error types derive from RuntimeError
        return []


def _run_variant(g, fx: dict, variant: str):
    e = load()["manifest"][variant]["engine"]
    n = fx["n"]
    if e["fn"] == "pagerank":
        p = e.get("personalization")
        pers = np.asarray(node_rule(p, n)) if p else None
        return g.pagerank(damping=float(e.get("damping", 0.85)),
                          directed=bool(e.get("directed", True)),
                          weighted=bool(e.get("weighted", False)), personalization=pers,
                          dangling=DANGLING[e.get("dangling", "personalized")],
                          loops=LOOPS[e.get("loops", "twice")])
    if e["fn"] == "eigenvector":
        vals, _, _ = target(g, e).eigenvector(mode=MODES[e.get("mode", "in")],
                                              weighted=bool(e.get("weighted", False)),
                                              scale=SCALES[e.get("scale", "max")],
                                              loops=LOOPS[e.get("loops", "twice")])
        return defined(vals)
    if e["fn"] == "twomode":
        # validation/bindings/twomode.py:130-159 (the eigenvector measure)
        if fx.get("type") is None:
            return []
        vals, _, _ = g.twomode_eigenvector(fx["type"])
        return defined(vals)
    if e["fn"] == "katz":
        mode, weighted, loops = e.get("mode", "in"), bool(e.get("weighted", False)), \
            e.get("loops", "once")
        alpha = relative(e, "alpha", g, mode, weighted, loops)
        b = e.get("beta", 1.0)
        beta = np.asarray(node_rule(b, n) if isinstance(b, str) else [float(b)])
        return g.katz(alpha=alpha, beta=beta, mode=MODES[mode], weighted=weighted,
                      loops=LOOPS[loops], normalized=bool(e.get("normalized", True)))
    if e["fn"] == "bonacich":
        mode, weighted, loops = e.get("mode", "out"), bool(e.get("weighted", False)), \
            e.get("loops", "ignore")
        t = target(g, e)
        exponent = relative(e, "exponent", t, "in" if mode == "out" else mode, weighted, loops)
        return t.bonacich(exponent=exponent, mode=MODES[mode], weighted=weighted,
                          loops=LOOPS[loops], rescale=bool(e.get("rescale", False)))
    if e["fn"] == "components":
        memb, _ = g.components(strong=e["kind"] == "strong")
        return [float(v) for v in memb]
    if e["fn"] == "centralization_eigenvector":
        # validation/bindings/roles.py:207-212: one value, NaN when undefined
        return [g.centralization_eigenvector(normalized=bool(e.get("normalized", True)))]
    if e["fn"] == "leading_eigen":
        # validation/bindings/groups.py:160-167,292-294,368-371
        memb, q, _ = g.leading_eigen(weighted=bool(e.get("weighted", False)))
        if e.get("output") == "membership":
            return [float(v) for v in memb]
        return [-1.0 if q != q else q]
    if e["fn"] == "hits":
        hubs, auths, _, _ = g.hits(weighted=bool(e.get("weighted", False)),
                                   loops=LOOPS[e.get("loops", "twice")],
                                   scale=HITS_SCALES[e.get("scale", "max")])
        return hubs if e["which"] == "hubs" else auths
    raise ValueError(e["fn"])


def canonical(values, mode: str):
    """validation/compare.py:40-60 for the modes on this path: values as
    given, or (partition) group labels renumbered by first appearance."""
    if mode == "partition":
        seen = {}
        return [None if v is None else float(seen.setdefault(v, len(seen))) for v in values]
    return list(values)


def agree_variant(ours, theirs, variant: str):
    """`agree` after putting both sides in the variant's comparison form."""
    spec = load()["manifest"][variant]
    mode = spec.get("compare", "values")
    return agree(canonical(list(ours), mode), canonical(list(theirs), mode), spec["tolerance"])


def agree(ours, theirs, tol: dict):
    """validation/compare.py:38-39: |a - b| <= abs + rel * max(|a|, |b|);
    an undefined golden value matches only NaN."""
    rel, abs_ = float(tol["rel"]), float(tol["abs"])
    if len(ours) != len(theirs):
        return False, f"length {len(ours)} != {len(theirs)}"
    for i, (a, b) in enumerate(zip(ours, theirs)):
        if b is None:
            if not math.isnan(a):
                return False, f"[{i}] {a} but golden undefined"
            continue
        if not abs(a - b) <= abs_ + rel * max(abs(a), abs(b)):
            return False, f"[{i}] {a!r} vs {b!r}"
    return True, ""
