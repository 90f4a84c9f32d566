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


def test_host_gnm_generator_matches_oracle(so):
    # The library's G(n, m) restates crates/engine/src/generate.rs:255-290;
    # both must give the same edges for the same stream.
    import numpy as np
    import knappnet_b200 as K
    from oracle import oracle as O
    for n, m, d, loops, seed in [(100, 300, False, False, 3), (50, 400, True, False, 4),
                                 (30, 200, False, True, 5), (20, 300, True, True, 6),
                                 (12, 60, False, False, 8)]:
        s, t = K.generate_gnm([n], [m], d, loops, seed)
        f, g = O.gnm(n, m, d, loops, seed, 0)
        assert np.array_equal(s, f) and np.array_equal(t, g)
    # a packed batch: graph k uses stream (seed, k) and global node numbers
    s, t = K.generate_gnm([10, 20], [15, 30], False, False, 9)
    f, g = O.gnm(20, 30, False, False, 9, 1)
    assert np.array_equal(s[15:], f + 10) and np.array_equal(t[15:], g + 10)


def test_power_law_sizes(so):
    import numpy as np
    import knappnet_b200 as K
    x = K.power_law_sizes(20000, 2.1, 50, 50000, 3)
    assert x.min() >= 50 and x.max() <= 50000
    # mean of the truncated continuous law, floored: about 275 - 0.5
    assert 240 < x.mean() < 310
    assert np.array_equal(x, K.power_law_sizes(20000, 2.1, 50, 50000, 3))


def test_projected_eigen_rejects_orders_beyond_twenty(so):
    """Checked before any device work: orders outside 0..20 fail, order 0
    succeeds with nothing to do."""
    import knappnet_b200 as K
    import numpy as np
    err = ctypes.create_string_buffer(K.ERR_LEN)
    a = np.zeros(441)
    assert K.lib().net_projected_eigen(21, K._ptr(a), K._ptr(a), K._ptr(a), err, K.ERR_LEN) != 0
    assert b"between 0 and 20" in err.value
    assert K.lib().net_projected_eigen(0, None, None, None, err, K.ERR_LEN) == 0


def test_tuning_keys_reject_bad_values(so):
    """Checked on the host: unknown keys and out-of-range values fail."""
    import knappnet_b200 as K
    L = K.lib()
    assert L.net_set_tuning(4, 13.0) != 0
    assert L.net_set_tuning(13, 9.0) != 0
    assert L.net_set_tuning(14, -2.0) != 0
    assert L.net_set_tuning(14, 0.5) != 0
    assert L.net_set_tuning(15, -1.0) != 0
    assert L.net_set_tuning(16, 2.0) != 0
    assert L.net_set_tuning(17, -1.0) != 0
    assert L.net_set_tuning(18, 0.0) != 0
    assert L.net_set_tuning(13, 0.0) == 0
    assert L.net_set_tuning(14, -1.0) == 0
    assert L.net_set_tuning(15, 0.0) == 0
    assert L.net_set_tuning(16, 0.0) == 0


def test_gather_calibration_checks_arguments_before_device_work(so):
    import knappnet_b200 as K
    L = K.lib()
    err = ctypes.create_string_buffer(K.ERR_LEN)
    r = ctypes.c_double()
    assert L.net_measure_gather(3, 1 << 20, ctypes.byref(r), err, K.ERR_LEN) != 0
    assert b"gather source" in err.value
    assert L.net_measure_gather(0, 100, ctypes.byref(r), err, K.ERR_LEN) != 0
    assert b"between 1024 and 2^31" in err.value
    assert L.net_measure_gather(0, 1 << 20, None, err, K.ERR_LEN) != 0
    assert b"null" in err.value
