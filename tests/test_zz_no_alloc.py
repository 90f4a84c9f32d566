"""The no-allocation PageRank entry point (net_pagerank_csr_static).

It is for callers that cannot call cudaMalloc, such as a host framework that
has reserved the device memory for its own allocator, or a path that must not
stall the device (cudaMalloc and cudaFree may synchronize it). Its scratch
lives in a static device array of the library, shared by all calls, so the
test runs two calls in a row and checks both against net_pagerank, the
allocating entry point, at the FP64 parity bar (L1 <= 1e-12). This file is
collected last so that a failure here stops a run only after every other
test has run.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import knappnet_b200 as K

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def entry():
    f = K.lib().net_pagerank_csr_static
    f.argtypes = [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                  ctypes.c_double, ctypes.c_double, ctypes.c_int64, ctypes.c_void_p,
                  ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p, ctypes.c_char_p,
                  ctypes.c_size_t]
    f.restype = ctypes.c_int32
    return f


def dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a).astype(dtype)).cuda()


def call(f, n, off, src, w, out, tol=1e-12):
    its = ctypes.c_int64()
    err = ctypes.create_string_buffer(K.ERR_LEN)
    status = f(n, ctypes.c_void_p(off.data_ptr()), ctypes.c_void_p(src.data_ptr()),
               None if w is None else ctypes.c_void_p(w.data_ptr()), 0.85, tol, 0,
               ctypes.c_void_p(out.data_ptr()), ctypes.byref(its), None, err, K.ERR_LEN)
    torch.cuda.synchronize()
    return status, its.value, err.value.decode()


@pytest.mark.parametrize("weighted", [True, False])
def test_static_scratch_pagerank_matches_allocating_entry_point(weighted):
    f = entry()
    g = K.generate_rmat(12, 16, seed=41, clean=True, lognormal=weighted, wseed=42)
    off, src, w = g.csr(1)  # rows = arcs into each node
    ref = g.pagerank(weighted=weighted)
    d_off, d_src = dev(off, np.int32), dev(src, np.int32)
    d_w = dev(w, np.float64) if weighted else None
    out = torch.empty(g.n, dtype=torch.float64, device="cuda")
    for _ in range(2):  # calls share the static scratch: both must be right
        out.fill_(-1.0)
        status, its, msg = call(f, g.n, d_off, d_src, d_w, out)
        assert status == 0, msg
        got = out.cpu().numpy()
        assert np.abs(got - ref).sum() <= 1e-12
        assert its > 0


def test_static_scratch_rejects_graphs_beyond_its_size():
    f = entry()
    n = (1 << 18) + 1
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    status, _, msg = call(f, n, dummy, dummy, None, out)
    assert status == 1
    assert "at most 262144 nodes" in msg
