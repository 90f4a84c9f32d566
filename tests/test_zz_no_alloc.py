"""The no-allocation PageRank entry point (net_pagerank_csr_static).

It is for callers that cannot call cudaMalloc, such as a host framework that
has reserved the device memory for its own allocator, or a path that must not
stall the device (cudaMalloc and cudaFree may synchronize it). Its scratch
lives in a static device array of the library, shared by all calls, so the
tests run calls back to back on graphs of different sizes (a larger graph
first, so leftovers of its scratch would show in the smaller one) and check
each against net_pagerank, the allocating entry point, at the FP64 parity bar
(L1 <= 1e-12); a graph of exactly the largest size the array holds is
checked against the CPU oracle. This file is collected last so that a
failure here stops a run only after every other test has run.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import knappnet_b200 as K
from oracle import oracle as O

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MAX_NODES = 1 << 18


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


def device_case(scale, weighted, seed):
    g = K.generate_rmat(scale, 16, seed=seed, clean=True, lognormal=weighted, wseed=seed + 1)
    off, src, w = g.csr(1)  # rows = arcs into each node
    ref = g.pagerank(weighted=weighted)
    arrays = (dev(off, np.int32), dev(src, np.int32), dev(w, np.float64) if weighted else None)
    n = g.n
    g.close()
    return n, arrays, ref


@pytest.mark.parametrize("weighted", [True, False])
def test_static_scratch_larger_then_smaller_graph(weighted):
    f = entry()
    cases = [device_case(12, weighted, 41), device_case(9, weighted, 43)]
    outs = {}
    for n, (d_off, d_src, d_w), ref in cases + cases:
        out = torch.full((n,), -1.0, dtype=torch.float64, device="cuda")
        status, its, msg = call(f, n, d_off, d_src, d_w, out)
        assert status == 0, msg
        got = out.cpu().numpy()
        assert np.abs(got - ref).sum() <= 1e-12
        assert its > 0
        if n in outs:  # the same graph again, after the other one: bit-identical
            assert np.array_equal(outs[n], got)
        outs[n] = got


def test_static_scratch_allocates_nothing_per_call():
    f = entry()
    n, (d_off, d_src, d_w), ref = device_case(10, True, 45)
    out = torch.empty(n, dtype=torch.float64, device="cuda")
    assert call(f, n, d_off, d_src, d_w, out)[0] == 0  # loads the module and its array
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        status, _, msg = call(f, n, d_off, d_src, d_w, out)
        assert status == 0, msg
    assert torch.cuda.mem_get_info()[0] == free0
    assert np.abs(out.cpu().numpy() - ref).sum() <= 1e-12


def test_static_scratch_at_its_largest_size_matches_oracle():
    f = entry()
    g = K.generate_rmat(18, 16, seed=47, clean=True, lognormal=True, wseed=48)
    assert g.n == MAX_NODES
    s, t, w = g.edges()
    off, src, wa = g.csr(1)
    og = O.Graph(g.n, s, t, w, True)
    ref = og.pagerank(weighted=True, tol=1e-12)
    out = torch.empty(g.n, dtype=torch.float64, device="cuda")
    status, its, msg = call(f, g.n, dev(off, np.int32), dev(src, np.int32),
                            dev(wa, np.float64), out)
    assert status == 0, msg
    # the oracle divides by a sequential sum; allow its own residual
    assert np.abs(out.cpu().numpy() - ref).sum() <= 1e-12 + abs(ref.sum() - 1.0)
    assert its == og.last_iters
    g.close()


def test_static_scratch_rejects_graphs_beyond_its_size():
    f = entry()
    n = MAX_NODES + 1
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    status, _, msg = call(f, n, dummy, dummy, None, out)
    assert status == 1
    assert "at most 262144 nodes" in msg


def test_static_scratch_checks_its_arrays():
    f = entry()
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    off = dev([0, 1, 2, 3], np.int32)
    # a source outside the graph: the kernel skips it and reports it
    status, _, msg = call(f, 3, off, dev([1, 7, 0], np.int32), None, out)
    assert status == 1 and "arc 1 has source 7, outside the graph's 3 nodes" in msg
    # a negative weight, as net_pagerank reports it
    status, _, msg = call(f, 3, off, dev([1, 2, 0], np.int32),
                          dev([1.0, 2.0, -0.5], np.float64), out)
    assert status == 1 and "arc 2 has negative weight -0.5" in msg
    assert "PageRank requires non-negative weights" in msg
    status, _, msg = call(f, 3, off, dev([1, 2, 0], np.int32),
                          dev([1.0, np.inf, 1.0], np.float64), out)
    assert status == 1 and "arc 1 has weight inf" in msg
    # offsets that decrease
    status, _, msg = call(f, 3, dev([0, 2, 1, 3], np.int32), dev([1, 2, 0], np.int32), None, out)
    assert status == 1 and "decrease after row 1" in msg
    # a NaN tolerance selects the default, as in net_pagerank
    good = dev([1, 2, 0], np.int32)
    status, its, msg = call(f, 3, off, good, None, out, tol=float("nan"))
    assert status == 0, msg
    assert np.allclose(out.cpu().numpy(), 1.0 / 3.0, atol=1e-15)
