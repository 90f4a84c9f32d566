"""CPU-only checks of the C ABI library: it builds, loads without a GPU, and
exports every function include/knappnet.h declares; host-only accessors
behave as the reference's (NULL handles give -1; freeing NULL is allowed)."""
from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "knappnet.h"


def declared_functions():
    text = HEADER.read_text()
    return re.findall(r"^NET_API\s+(?:int32_t|int64_t|void)\s+(net_\w+)\(", text, re.M)


@pytest.fixture(scope="module")
def so():
    from knappnet_b200 import build
    return build.build()


def test_header_declares_the_reference_entry_points():
    names = set(declared_functions())
    for fn in ("net_graph_new", "net_graph_free", "net_graph_node_count", "net_graph_edge_count",
               "net_degree", "net_pagerank", "net_eigenvector"):
        assert fn in names


def test_library_exports_every_declared_symbol(so):
    lib = ctypes.CDLL(str(so))
    missing = [fn for fn in declared_functions() if not hasattr(lib, fn)]
    assert not missing, missing


def test_null_handles(so):
    import knappnet_b200 as K
    L = K.lib()
    assert L.net_graph_node_count(None) == -1
    assert L.net_graph_edge_count(None) == -1
    assert L.net_graph_arc_count(None, 0) == -1
    L.net_graph_free(None)
    err = ctypes.create_string_buffer(256)
    out = (ctypes.c_double * 4)()
    assert L.net_degree(None, 3, 1, 0, out, err, 256) == 1
    assert b"null" in err.value
    assert L.net_pagerank(None, 0.85, 1, 0, None, 0, 0, 0.0, 0, 0, out, err, 256) == 1
    assert b"null" in err.value


def test_reference_signatures_match_header():
    # net_pagerank and net_eigenvector keep the reference's parameter lists
    # (crates/capi/include/netcapi.h:455-467).
    text = " ".join(HEADER.read_text().split())
    assert ("net_pagerank(const GraphHandle *h, double damping, int32_t directed, int32_t "
            "weighted, const double *personalization, int32_t dangling, int32_t loops, double "
            "tol, int64_t max_iter, int32_t threads, double *out, char *err, size_t err_len)"
            in text)
    assert ("net_eigenvector(const GraphHandle *h, int32_t mode, int32_t weighted, int32_t "
            "scale, int32_t loops, double tol, int64_t max_iter, int32_t threads, double *out, "
            "double *eigenvalue, int32_t *connected, char *err, size_t err_len)" in text)
