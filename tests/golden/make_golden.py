"""Packs the reference's validation fixtures and golden values for the
spectral-centrality path into tests/golden/spectral_golden.json.

The reference ships 28 small fixture networks (validation/fixtures/<name>/
edges.csv + meta.json) and, per fixture, golden answers written by
independent oracles (validation/golden/<oracle>/<fixture>/<variant>.csv):
"definition" (dense linear algebra) and "networkx" (NetworkX 3.7). The
variants and their options and tolerances come from
validation/manifest.d/spectral.yaml (PageRank) and topography.yaml
(eigenvector centrality).

The GPU box has no copy of the reference, so the tests read this packed
file. Regenerate it with

    python tests/golden/make_golden.py --reference <path of the reference checkout>
"""
from __future__ import annotations

import argparse
import csv
import json
import math
from pathlib import Path

import yaml

HERE = Path(__file__).resolve().parent

# Variants on the spectral-centrality path: PageRank, Katz, Bonacich power
# centrality and hubs and authorities (spectral.yaml), eigenvector centrality
# and the components it is computed on (topography.yaml), eigenvector
# centralization (roles.yaml).
# The sna and UCINET variants read the network through net_graph_simplify
# first; two-mode eigenvector centrality (twomode.yaml) needs the node types
# the two-mode fixtures record; Newman's leading eigenvector communities
# (groups.yaml) divide by the signs of a leading eigenvector.
VARIANTS = {
    "spectral.yaml": ["pagerank", "pagerank_networkx", "pagerank_weighted",
                      "pagerank_personalized", "pagerank_personalized_networkx",
                      "pagerank_uniform_dangling", "pagerank_undirected",
                      "katz", "katz_weighted", "katz_igraph", "katz_exogenous",
                      "bonacich", "bonacich_negative", "bonacich_unit", "bonacich_rescale",
                      "bonacich_sna",
                      "hits_authorities", "hits_hubs", "hits_authorities_networkx",
                      "hits_hubs_networkx"],
    "topography.yaml": ["eigenvector", "eigenvector_networkx", "eigenvector_weighted",
                        "eigenvector_weighted_networkx", "eigenvector_undirected",
                        "eigenvector_sna", "eigenvector_ucinet",
                        "components_weak", "components_strong"],
    "roles.yaml": ["centralization_eigenvector"],
    "twomode.yaml": ["twomode_eigenvector"],
    "groups.yaml": ["leading_eigen", "leading_eigen_membership", "leading_eigen_weighted"],
}
ORACLES = ["definition", "networkx"]


def read_values(path: Path):
    if not path.exists():
        return None
    out = []
    with open(path) as fh:
        next(fh)
        for line in fh:
            parts = line.split()
            if not parts or parts[0] == "NA":
                out.append(None)
            else:
                v = float(parts[0])
                out.append(None if math.isnan(v) else v)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True,
                    help="root of the reference checkout (holds validation/)")
    ap.add_argument("--out", default=str(HERE / "spectral_golden.json"))
    args = ap.parse_args()
    val = Path(args.reference) / "validation"

    manifest = {}
    for fname, names in VARIANTS.items():
        entries = yaml.safe_load((val / "manifest.d" / fname).read_text())
        for name in names:
            e = entries[name]
            manifest[name] = {
                "engine": e["engine"],
                "applies_to": e.get("applies_to", "any"),
                "requires_weights": bool(e.get("requires_weights", False)),
                "tolerance": e["tolerance"],
                "compare": e.get("compare", "values"),
                "source": f"validation/manifest.d/{fname}",
            }

    fixtures = {}
    golden = {}
    for d in sorted(p for p in (val / "fixtures").iterdir() if (p / "meta.json").exists()):
        meta = json.loads((d / "meta.json").read_text())
        src, tgt, w = [], [], []
        with open(d / "edges.csv", newline="") as fh:
            for row in csv.DictReader(fh):
                src.append(int(row["from"]))
                tgt.append(int(row["to"]))
                if meta["weighted"]:
                    w.append(float(row["weight"]))
        fixtures[d.name] = {
            "n": meta["n"], "directed": meta["directed"], "weighted": meta["weighted"],
            "tags": meta.get("tags", []), "type": meta.get("type"), "src": src, "tgt": tgt,
            "w": w if meta["weighted"] else None,
        }
        g = {}
        for variant in manifest:
            per = {}
            for oracle in ORACLES:
                vals = read_values(val / "golden" / oracle / d.name / f"{variant}.csv")
                if vals is not None:
                    per[oracle] = vals
            if per:
                g[variant] = per
        golden[d.name] = g

    versions = {o: (val / "golden" / o / "VERSION").read_text().strip() for o in ORACLES}
    doc = {
        "about": "validation fixtures and golden values of the reference engine "
                 "(validation/fixtures, validation/golden/{definition,networkx}) for "
                 "PageRank, Katz, Bonacich power, HITS, eigenvector centrality (one- and "
                 "two-mode), components, eigenvector centralization and leading eigenvector "
                 "communities; generated "
                 "by make_golden.py",
        "oracle_versions": versions,
        "manifest": manifest,
        "fixtures": fixtures,
        "golden": golden,
    }
    Path(args.out).write_text(json.dumps(doc, separators=(",", ":")))
    n_vals = sum(len(v) for g in golden.values() for v in g.values())
    print(f"wrote {args.out}: {len(fixtures)} fixtures, {n_vals} golden vectors")


if __name__ == "__main__":
    main()
