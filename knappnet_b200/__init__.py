"""knappnet B200: the reference engine's spectral-centrality path on an NVIDIA
B200 (sm_100a), behind the reference's C ABI.

The compute lives in the CUDA library libknappnet_b200.so (C ABI declared in
include/knappnet.h). This module is a thin ctypes binding with the same
calls and argument meaning as the reference's ctypes bindings
(validation/bindings/spectral.py, topography.py): a graph handle, then
degree, PageRank and eigenvector centrality on it.

There is no CPU fallback: if the library is missing or cannot be loaded,
importing `lib()` raises.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libknappnet_b200.so"
ERR_LEN = 1024

PREC_FP64, PREC_MIXED, PREC_FP32 = 0, 1, 2

_lib = None


class EngineError(RuntimeError):
    """A call of the C ABI returned a failure status."""


class NetBatchInfo(ctypes.Structure):
    _fields_ = [("seconds", ctypes.c_double), ("sweeps", ctypes.c_int64),
                ("sweeps_fp32", ctypes.c_int64), ("column_iterations", ctypes.c_int64),
                ("max_column_iterations", ctypes.c_int64), ("kernel_launches", ctypes.c_int32),
                ("refined", ctypes.c_int32), ("sweep_seconds", ctypes.c_double),
                ("column_iterations_fp32", ctypes.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class NetSolveInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int64), ("iterations_fp32", ctypes.c_int64),
                ("change", ctypes.c_double), ("seconds", ctypes.c_double),
                ("converged", ctypes.c_int32), ("kernel_launches", ctypes.c_int32),
                ("eigenvalue", ctypes.c_double), ("connected", ctypes.c_int32),
                ("sweep_kernel", ctypes.c_int32), ("long_row", ctypes.c_int32),
                ("hot_columns", ctypes.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def lib() -> ctypes.CDLL:
    """The loaded CUDA library (built in-tree by knappnet_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("KNAPPNET_LIB", LIB_PATH))
    if not path.exists():
        raise EngineError(f"{path} is missing: build it with `python -m knappnet_b200.build`")
    L = ctypes.CDLL(str(path))
    i32, i64, u64, f64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double
    vp, cp, sz = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t
    h = ctypes.c_void_p
    info_p = ctypes.POINTER(NetSolveInfo)
    L.net_frame_graph.argtypes = [i64, vp, vp, vp, vp, i64, i32, ctypes.POINTER(h), vp,
                                  ctypes.POINTER(i64), cp, sz]
    L.net_frame_graph.restype = i32
    L.net_frame_egos.argtypes = [i64, vp, vp, vp, vp, i64, i32, vp, vp, i64, ctypes.POINTER(h),
                                 vp, vp, vp, ctypes.POINTER(i64), cp, sz]
    L.net_frame_egos.restype = i32
    L.net_projected_eigen.argtypes = [i64, vp, vp, vp, cp, sz]
    L.net_projected_eigen.restype = i32
    L.net_graph_new.argtypes = [i64, vp, vp, vp, i64, i32, ctypes.POINTER(h), cp, sz]
    L.net_graph_new.restype = i32
    L.net_graph_free.argtypes = [h]
    L.net_graph_free.restype = None
    L.net_graph_node_count.argtypes = [h]
    L.net_graph_node_count.restype = i64
    L.net_graph_edge_count.argtypes = [h]
    L.net_graph_edge_count.restype = i64
    L.net_degree.argtypes = [h, i32, i32, i32, vp, cp, sz]
    L.net_degree.restype = i32
    L.net_pagerank.argtypes = [h, f64, i32, i32, vp, i32, i32, f64, i64, i32, vp, cp, sz]
    L.net_pagerank.restype = i32
    L.net_eigenvector.argtypes = [h, i32, i32, i32, i32, f64, i64, i32, vp,
                                  ctypes.POINTER(f64), ctypes.POINTER(i32), cp, sz]
    L.net_eigenvector.restype = i32
    L.net_graph_simplify.argtypes = [h, i32, i32, ctypes.POINTER(h), cp, sz]
    L.net_graph_simplify.restype = i32
    L.net_twomode_eigenvector.argtypes = [h, vp, f64, i64, i32, vp, ctypes.POINTER(f64),
                                          ctypes.POINTER(i32), cp, sz]
    L.net_twomode_eigenvector.restype = i32
    L.net_leading_eigen.argtypes = [h, i32, vp, ctypes.POINTER(f64), ctypes.POINTER(i64), cp, sz]
    L.net_leading_eigen.restype = i32
    L.net_components.argtypes = [h, i32, vp, ctypes.POINTER(i64), cp, sz]
    L.net_components.restype = i32
    L.net_centralization.argtypes = [h, i32, i32, i32, i32, i32, i32, ctypes.POINTER(f64), cp, sz]
    L.net_centralization.restype = i32
    L.net_katz.argtypes = [h, f64, vp, i64, i32, i32, i32, i32, f64, i64, i32, vp, cp, sz]
    L.net_katz.restype = i32
    L.net_bonacich_power.argtypes = [h, f64, i32, i32, i32, i32, f64, i64, i32, vp, cp, sz]
    L.net_bonacich_power.restype = i32
    L.net_hits.argtypes = [h, i32, i32, i32, f64, i64, i32, vp, vp, ctypes.POINTER(f64),
                           ctypes.POINTER(i32), cp, sz]
    L.net_hits.restype = i32
    L.net_pagerank_ex.argtypes = [h, f64, i32, i32, vp, i32, i32, f64, i64, i32, vp, info_p,
                                  cp, sz]
    L.net_pagerank_ex.restype = i32
    L.net_pagerank_device.argtypes = [h, f64, i32, i32, vp, i32, i32, f64, i64, i32, vp, info_p,
                                      cp, sz]
    L.net_pagerank_device.restype = i32
    L.net_eigenvector_ex.argtypes = [h, i32, i32, i32, i32, f64, i64, i32, vp,
                                     ctypes.POINTER(f64), ctypes.POINTER(i32), info_p, cp, sz]
    L.net_eigenvector_ex.restype = i32
    binfo_p = ctypes.POINTER(NetBatchInfo)
    L.net_pagerank_batch.argtypes = [h, f64, i32, i32, vp, i64, i32, i32, f64, i64, i32, vp,
                                     binfo_p, cp, sz]
    L.net_pagerank_batch.restype = i32
    L.net_pagerank_batch_device.argtypes = [h, f64, i32, i32, vp, i64, i32, i32, f64, i64, i32,
                                            vp, binfo_p, cp, sz]
    L.net_pagerank_batch_device.restype = i32
    L.net_pagerank_graphs.argtypes = [h, i64, vp, f64, i32, i32, vp, i32, i32, f64, i64, vp, vp,
                                      info_p, cp, sz]
    L.net_pagerank_graphs.restype = i32
    L.net_generate_gnm.argtypes = [i64, vp, vp, i32, i32, u64, vp, vp, cp, sz]
    L.net_generate_gnm.restype = i32
    L.net_power_law_sizes.argtypes = [i64, f64, f64, f64, u64, vp, cp, sz]
    L.net_power_law_sizes.restype = i32
    L.net_pagerank_weights_device.argtypes = [h, vp, f64, i32, vp, i32, i32, f64, i64, i32, vp,
                                              info_p, cp, sz]
    L.net_pagerank_weights_device.restype = i32
    L.net_pagerank_grad_device.argtypes = [h, vp, vp, vp, f64, i32, vp, i32, i32, f64, i64, vp,
                                           vp, info_p, cp, sz]
    L.net_pagerank_grad_device.restype = i32
    L.net_graph_new_device.argtypes = [i64, vp, vp, vp, vp, i64, i32, ctypes.POINTER(h), cp, sz]
    L.net_graph_new_device.restype = i32
    L.net_graph_arc_count.argtypes = [h, i32]
    L.net_graph_arc_count.restype = i64
    L.net_graph_csr.argtypes = [h, i32, vp, vp, vp, vp, cp, sz]
    L.net_graph_csr.restype = i32
    L.net_graph_edges.argtypes = [h, vp, vp, vp, cp, sz]
    L.net_graph_edges.restype = i32
    L.net_generate_rmat.argtypes = [i32, i64, f64, f64, f64, u64, i32, i32, i32, u64,
                                    ctypes.POINTER(h), ctypes.POINTER(i64), cp, sz]
    L.net_generate_rmat.restype = i32
    L.net_sweep_timing.argtypes = [i32, ctypes.POINTER(i64), ctypes.POINTER(f64),
                                   ctypes.POINTER(f64)]
    L.net_sweep_timing.restype = i32
    L.net_set_sweep_timing.argtypes = [i32]
    L.net_set_sweep_timing.restype = None
    L.net_measure_gather.argtypes = [i32, i64, ctypes.POINTER(f64), cp, sz]
    L.net_measure_gather.restype = i32
    L.net_set_tuning.argtypes = [i32, f64]
    L.net_set_tuning.restype = i32
    L.net_device_sync.argtypes = [cp, sz]
    L.net_device_sync.restype = i32
    L.net_shard_bounds.argtypes = [h, i32, i32, i32, i32, vp, cp, sz]
    L.net_shard_bounds.restype = i32
    L.net_shard_new.argtypes = [h, f64, i32, i32, vp, i32, i32, vp, i32, i32, ctypes.POINTER(h),
                                ctypes.POINTER(i64), cp, sz]
    L.net_shard_new.restype = i32
    L.net_shard_sweep.argtypes = [h, vp, vp, cp, sz]
    L.net_shard_sweep.restype = i32
    L.net_shard_finish.argtypes = [h, vp, ctypes.POINTER(f64), vp, cp, sz]
    L.net_shard_finish.restype = i32
    L.net_shard_scores.argtypes = [h, vp, i32, vp, cp, sz]
    L.net_shard_scores.restype = i32
    L.net_shard_restart.argtypes = [h, vp, cp, sz]
    L.net_shard_restart.restype = i32
    L.net_shard_free.argtypes = [h]
    L.net_shard_free.restype = None
    _lib = L
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _check(status: int, err) -> None:
    if status:
        raise EngineError(err.value.decode(errors="replace"))


class Graph:
    """A graph handle in GPU memory (net_graph_new / net_graph_free)."""

    def __init__(self, n, src=None, tgt=None, weights=None, directed=True, _handle=None,
                 _m=None, _weighted=None):
        self.n = int(n)
        self.directed = bool(directed)
        if _handle is not None:
            self.h = _handle
            self.m = int(_m)
            self.weighted = bool(_weighted)
            return
        s = np.ascontiguousarray(src, dtype=np.int64)
        t = np.ascontiguousarray(tgt, dtype=np.int64)
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        self.m = len(s)
        self.weighted = w is not None
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_graph_new(self.n, _ptr(s), _ptr(t), _ptr(w), self.m, int(directed),
                                   ctypes.byref(h), err, ERR_LEN), err)
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.net_graph_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def node_count(self) -> int:
        return int(lib().net_graph_node_count(self.h))

    def edge_count(self) -> int:
        return int(lib().net_graph_edge_count(self.h))

    def csr(self, which: int = 0, edges: bool = False):
        """(off, tgt, w) of the out (0), in (1) or undirected (2) CSR, and the
        input edge of each arc when edges=True."""
        arcs = int(lib().net_graph_arc_count(self.h, which if which != 2 else 0))
        if which == 2:
            arcs = -1
        off = np.zeros(self.n + 1, dtype=np.uint32)
        err = ctypes.create_string_buffer(ERR_LEN)
        if arcs < 0:  # undirected rows: size known after the offsets
            _check(lib().net_graph_csr(self.h, which, _ptr(off), None, None, None, err, ERR_LEN),
                   err)
            arcs = int(off[-1])
        tgt = np.zeros(max(arcs, 1), dtype=np.uint32)
        eid = np.zeros(max(arcs, 1), dtype=np.uint32) if edges else None
        w = np.zeros(max(arcs, 1), dtype=np.float64) if self.weighted else None
        _check(lib().net_graph_csr(self.h, which, _ptr(off), _ptr(tgt), _ptr(eid), _ptr(w), err,
                                   ERR_LEN), err)
        out = (off.astype(np.uint64), tgt[:arcs], None if w is None else w[:arcs])
        if edges:
            return out + (eid[:arcs],)
        return out

    def edges(self):
        s = np.zeros(max(self.m, 1), dtype=np.int64)
        t = np.zeros(max(self.m, 1), dtype=np.int64)
        w = np.zeros(max(self.m, 1)) if self.weighted else None
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_graph_edges(self.h, _ptr(s), _ptr(t), _ptr(w), err, ERR_LEN), err)
        return s[: self.m], t[: self.m], (None if w is None else w[: self.m])

    def degree(self, mode=3, loops=True, weighted=False):
        out = np.zeros(max(self.n, 1))
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_degree(self.h, mode, int(loops), int(weighted), _ptr(out), err,
                                ERR_LEN), err)
        return out[: self.n]

    def pagerank(self, damping=0.85, directed=True, weighted=False, personalization=None,
                 dangling=0, loops=0, tol=0.0, max_iter=0, threads=0, precision=PREC_FP64):
        vals, _ = self.pagerank_ex(damping, directed, weighted, personalization, dangling, loops,
                                   tol, max_iter, precision)
        return vals

    def pagerank_ex(self, damping=0.85, directed=True, weighted=False, personalization=None,
                    dangling=0, loops=0, tol=0.0, max_iter=0, precision=PREC_FP64, out=None):
        if out is None:
            out = np.zeros(max(self.n, 1))
        p = None if personalization is None else np.ascontiguousarray(personalization,
                                                                       dtype=np.float64)
        info = NetSolveInfo()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_pagerank_ex(self.h, damping, int(directed), int(weighted), _ptr(p),
                                     dangling, loops, tol, max_iter, precision, _ptr(out),
                                     ctypes.byref(info), err, ERR_LEN), err)
        return out[: self.n], info

    def pagerank_device(self, out_ptr: int, damping=0.85, directed=True, weighted=False,
                        personalization_ptr=None, dangling=0, loops=0, tol=0.0, max_iter=0,
                        precision=PREC_FP64):
        """net_pagerank_device: scores written to device memory at out_ptr (n
        doubles, e.g. a torch CUDA tensor's data_ptr()); the optional teleport
        vector is read from device memory."""
        info = NetSolveInfo()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_pagerank_device(self.h, damping, int(directed), int(weighted),
                                         personalization_ptr, dangling, loops, tol, max_iter,
                                         precision, ctypes.c_void_p(out_ptr), ctypes.byref(info),
                                         err, ERR_LEN), err)
        return info

    def shard_bounds(self, parts, directed=True, weighted=False, loops=0):
        """net_shard_bounds: parts + 1 row boundaries of PageRank's pull
        operator giving each part about an equal share of rows plus arcs."""
        b = np.zeros(int(parts) + 1, dtype=np.int64)
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_shard_bounds(self.h, int(directed), int(weighted), loops, int(parts),
                                      _ptr(b), err, ERR_LEN), err)
        return b

    def pagerank_batch(self, personalization, damping=0.85, directed=True, weighted=False,
                       dangling=0, loops=0, tol=0.0, max_iter=0, precision=PREC_FP64):
        """Personalised PageRank for every row of `personalization` (shape
        (batch, n)); returns scores of the same shape and the NetBatchInfo."""
        P = np.ascontiguousarray(personalization, dtype=np.float64)
        if P.ndim != 2 or P.shape[1] != self.n:
            raise ValueError("personalization must have shape (batch, n)")
        # written with zeros first: copying scores into untouched pages
        # would fault them in during the device-to-host copy, which is slower
        out = np.zeros_like(P)
        info = NetBatchInfo()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_pagerank_batch(self.h, damping, int(directed), int(weighted), _ptr(P),
                                        P.shape[0], dangling, loops, tol, max_iter, precision,
                                        _ptr(out), ctypes.byref(info), err, ERR_LEN), err)
        return out, info

    def pagerank_batch_device(self, p_ptr: int, batch: int, out_ptr: int, damping=0.85,
                              directed=True, weighted=False, dangling=0, loops=0, tol=0.0,
                              max_iter=0, precision=PREC_FP64):
        """net_pagerank_batch_device: teleport vectors and scores in device
        memory (batch x n, vector c at offset c * n); returns NetBatchInfo."""
        info = NetBatchInfo()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_pagerank_batch_device(self.h, damping, int(directed), int(weighted),
                                               ctypes.c_void_p(p_ptr), batch, dangling, loops,
                                               tol, max_iter, precision,
                                               ctypes.c_void_p(out_ptr), ctypes.byref(info), err,
                                               ERR_LEN), err)
        return info

    def pagerank_graphs(self, node_offsets, damping=0.85, directed=True, weighted=False,
                        personalization=None, dangling=0, loops=0, tol=0.0, max_iter=0):
        """PageRank of every graph packed in this handle (graph k on nodes
        node_offsets[k]..node_offsets[k+1]-1): scores, per-graph iteration
        counts, NetSolveInfo."""
        off = np.ascontiguousarray(node_offsets, dtype=np.int64)
        count = len(off) - 1
        p = None if personalization is None else np.ascontiguousarray(personalization,
                                                                       dtype=np.float64)
        out = np.zeros(max(self.n, 1))
        its = np.zeros(max(count, 1), dtype=np.int64)
        info = NetSolveInfo()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_pagerank_graphs(self.h, count, _ptr(off), damping, int(directed),
                                         int(weighted), _ptr(p), dangling, loops, tol, max_iter,
                                         _ptr(out), _ptr(its), ctypes.byref(info), err, ERR_LEN),
               err)
        return out[: self.n], its[:count], info

    def pagerank_reference_call(self, damping=0.85, directed=True, weighted=False,
                                personalization=None, dangling=0, loops=0, tol=0.0, max_iter=0,
                                threads=0):
        """net_pagerank with the reference's exact signature."""
        out = np.zeros(max(self.n, 1))
        p = None if personalization is None else np.ascontiguousarray(personalization,
                                                                       dtype=np.float64)
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_pagerank(self.h, damping, int(directed), int(weighted), _ptr(p),
                                  dangling, loops, tol, max_iter, threads, _ptr(out), err,
                                  ERR_LEN), err)
        return out[: self.n]

    def katz(self, alpha=0.1, beta=1.0, mode=2, weighted=False, loops=1, normalized=True,
             tol=0.0, max_iter=0, threads=0):
        """net_katz: Katz centrality; beta is one value or n values."""
        b = np.ascontiguousarray(np.atleast_1d(beta), dtype=np.float64)
        out = np.zeros(max(self.n, 1))
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_katz(self.h, alpha, _ptr(b), len(b), mode, int(weighted), loops,
                              int(normalized), tol, max_iter, threads, _ptr(out), err, ERR_LEN),
               err)
        return out[: self.n]

    def bonacich(self, exponent=1.0, mode=1, weighted=False, loops=2, rescale=False, tol=0.0,
                 max_iter=0, threads=0):
        """net_bonacich_power: Bonacich power centrality."""
        out = np.zeros(max(self.n, 1))
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_bonacich_power(self.h, exponent, mode, int(weighted), loops,
                                        int(rescale), tol, max_iter, threads, _ptr(out), err,
                                        ERR_LEN), err)
        return out[: self.n]

    def hits(self, weighted=False, loops=0, scale=0, tol=0.0, max_iter=0, threads=0):
        """net_hits: hubs, authorities, the largest eigenvalue of A^T A and
        whether the leading singular value is simple."""
        hubs = np.zeros(max(self.n, 1))
        auths = np.zeros(max(self.n, 1))
        val = ctypes.c_double()
        uniq = ctypes.c_int32()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_hits(self.h, int(weighted), loops, scale, tol, max_iter, threads,
                              _ptr(hubs), _ptr(auths), ctypes.byref(val), ctypes.byref(uniq),
                              err, ERR_LEN), err)
        return hubs[: self.n], auths[: self.n], val.value, bool(uniq.value)

    def simplify(self, undirected=False, keep=0):
        """The adjacency-matrix reading (net_graph_simplify): loops dropped,
        parallel edges merged keeping the largest (keep 0) or smallest
        (keep 1) weight; undirected symmetrizes a directed graph."""
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_graph_simplify(self.h, int(bool(undirected)), int(keep), ctypes.byref(h),
                                        err, ERR_LEN), err)
        m = int(lib().net_graph_edge_count(h))
        return Graph(self.n, directed=self.directed and not undirected, _handle=h, _m=m,
                     _weighted=self.weighted)

    def twomode_eigenvector(self, types, tol=0.0, max_iter=0):
        """Two-mode eigenvector centrality (net_twomode_eigenvector):
        (scores, largest singular value, connected)."""
        t = np.ascontiguousarray(types, dtype=np.int32)
        out = np.zeros(max(self.n, 1))
        val = ctypes.c_double()
        conn = ctypes.c_int32()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_twomode_eigenvector(self.h, _ptr(t), tol, max_iter, 0, _ptr(out),
                                             ctypes.byref(val), ctypes.byref(conn), err,
                                             ERR_LEN), err)
        return out[: self.n], val.value, bool(conn.value)

    def leading_eigen(self, weighted=False):
        """Newman's leading eigenvector communities (net_leading_eigen):
        (labels, modularity, divisions)."""
        memb = np.zeros(max(self.n, 1), dtype=np.int64)
        q = ctypes.c_double()
        splits = ctypes.c_int64()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_leading_eigen(self.h, int(bool(weighted)), _ptr(memb), ctypes.byref(q),
                                       ctypes.byref(splits), err, ERR_LEN), err)
        return memb[: self.n], q.value, splits.value

    def components(self, strong=False):
        """Weak or strong components (net_components): labels numbered in
        order of each component's lowest node, and their count."""
        memb = np.zeros(max(self.n, 1), dtype=np.int32)
        cnt = ctypes.c_int64()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_components(self.h, int(bool(strong)), _ptr(memb), ctypes.byref(cnt),
                                    err, ERR_LEN), err)
        return memb[: self.n], cnt.value

    def centralization(self, measure=3, mode=3, loops=True, normalized=True, convention=0):
        """Freeman centralization (net_centralization); this library
        provides the eigenvector measure (3) under the igraph convention."""
        out = ctypes.c_double()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_centralization(self.h, measure, mode, int(loops), int(normalized),
                                        convention, 0, ctypes.byref(out), err, ERR_LEN), err)
        return out.value

    def centralization_eigenvector(self, normalized=True):
        return self.centralization(3, 3, True, normalized, 0)

    def eigenvector(self, mode=2, weighted=False, scale=0, loops=0, tol=0.0, max_iter=0,
                    threads=0, precision=0):
        vals, info = self.eigenvector_ex(mode, weighted, scale, loops, tol, max_iter, precision)
        return vals, info.eigenvalue, bool(info.connected)

    def eigenvector_ex(self, mode=2, weighted=False, scale=0, loops=0, tol=0.0, max_iter=0,
                       precision=0):
        out = np.zeros(max(self.n, 1))
        val = ctypes.c_double()
        conn = ctypes.c_int32()
        info = NetSolveInfo()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_eigenvector_ex(self.h, mode, int(weighted), scale, loops, tol, max_iter,
                                        precision, _ptr(out), ctypes.byref(val),
                                        ctypes.byref(conn), ctypes.byref(info), err, ERR_LEN),
               err)
        info.eigenvalue = val.value
        info.connected = conn.value
        return out[: self.n], info


def _stream_ptr(t):
    """The CUDA stream handle of torch's current stream on t's device (None
    for a CPU tensor or a plain pointer)."""
    if hasattr(t, "is_cuda") and t.is_cuda:
        import torch
        return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)
    return None


def _dev_ptr(t, count=None):
    """A device pointer from a raw address or a CUDA tensor; a tensor must
    be contiguous float64 on a GPU and hold at least `count` values."""
    if isinstance(t, int):
        return ctypes.c_void_p(t)
    import torch
    if not t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous():
        raise ValueError("the buffer must be a contiguous float64 CUDA tensor")
    if count is not None and t.numel() < count:
        raise ValueError(f"the buffer holds {t.numel()} values; {count} are needed")
    return ctypes.c_void_p(t.data_ptr())


class Shard:
    """One rank's row shard of a graph's PageRank split over several GPUs by
    rows (net_shard_new): `sweep` writes this rank's payload, `finish` takes
    the payloads of all ranks gathered in rank order and returns the L1
    change, `scores` reads the iterate. Buffers are CUDA tensors (or device
    pointers); calls run on torch's current stream of the tensor's device."""

    def __init__(self, graph, bounds, rank, damping=0.85, directed=True, weighted=False,
                 personalization_ptr=None, dangling=0, loops=0):
        b = np.ascontiguousarray(bounds, dtype=np.int64)
        self.parts = len(b) - 1
        self.rank = int(rank)
        self.n = graph.n
        self.bounds = b
        self._graph = graph  # the shard reads the graph's operator
        h = ctypes.c_void_p()
        plen = ctypes.c_int64()
        err = ctypes.create_string_buffer(ERR_LEN)
        pp = None if personalization_ptr is None else ctypes.c_void_p(personalization_ptr)
        _check(lib().net_shard_new(graph.h, damping, int(directed), int(weighted), pp, dangling,
                                   loops, _ptr(b), self.parts, self.rank, ctypes.byref(h),
                                   ctypes.byref(plen), err, ERR_LEN), err)
        self.h = h
        self.payload_len = int(plen.value)

    def sweep(self, payload):
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_shard_sweep(self.h, _dev_ptr(payload, self.payload_len),
                                     _stream_ptr(payload), err, ERR_LEN), err)

    def finish(self, gathered) -> float:
        change = ctypes.c_double()
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_shard_finish(self.h, _dev_ptr(gathered, self.parts * self.payload_len),
                                      ctypes.byref(change), _stream_ptr(gathered), err,
                                      ERR_LEN), err)
        return change.value

    def restart(self, like=None):
        """Back to the uniform iterate (on torch's current stream of `like`'s
        device, if given)."""
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_shard_restart(self.h, _stream_ptr(like), err, ERR_LEN), err)

    def scores(self):
        out = np.zeros(self.n)
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_shard_scores(self.h, _ptr(out), 0, None, err, ERR_LEN), err)
        return out

    def scores_device(self, out):
        err = ctypes.create_string_buffer(ERR_LEN)
        _check(lib().net_shard_scores(self.h, _dev_ptr(out, self.n), 1, _stream_ptr(out), err,
                                      ERR_LEN), err)

    def close(self):
        if getattr(self, "h", None) is not None and _lib is not None:
            _lib.net_shard_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


def generate_rmat(scale, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=1, clean=True,
                  symmetrize=False, lognormal=False, wseed=2) -> Graph:
    """An R-MAT graph generated and built on the device (net_generate_rmat)."""
    h = ctypes.c_void_p()
    m = ctypes.c_int64()
    err = ctypes.create_string_buffer(ERR_LEN)
    _check(lib().net_generate_rmat(scale, edge_factor, a, b, c, seed, int(clean), int(symmetrize),
                                   int(lognormal), wseed, ctypes.byref(h), ctypes.byref(m), err,
                                   ERR_LEN), err)
    return Graph(1 << scale, directed=not symmetrize, _handle=h, _m=m.value, _weighted=lognormal)


def frame_graph(n, src, tgt, weights=None, missing=None, directed=True):
    """The graph of a resolved edge table's observed rows (net_frame_graph):
    returns (Graph, table row of each graph edge)."""
    s = np.ascontiguousarray(src, dtype=np.int64)
    t = np.ascontiguousarray(tgt, dtype=np.int64)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    miss = None if missing is None else np.ascontiguousarray(missing, dtype=np.uint8)
    m = len(s)
    rows = np.zeros(max(m, 1), dtype=np.int64)
    cnt = ctypes.c_int64()
    h = ctypes.c_void_p()
    err = ctypes.create_string_buffer(ERR_LEN)
    _check(lib().net_frame_graph(int(n), _ptr(s), _ptr(t), _ptr(w), _ptr(miss), m, int(directed),
                                 ctypes.byref(h), _ptr(rows), ctypes.byref(cnt), err, ERR_LEN), err)
    return (Graph(int(n), directed=directed, _handle=h, _m=cnt.value, _weighted=w is not None),
            rows[: cnt.value])


def frame_egos(n, src, tgt, node_ego, edge_ego, egos, weights=None, missing=None, directed=True):
    """Every ego network of a resolved table packed into one graph
    (net_frame_egos): returns (Graph, node_offsets, table node of each packed
    node, table row of each packed edge). edge_ego None: every row takes its
    source's ego."""
    s = np.ascontiguousarray(src, dtype=np.int64)
    t = np.ascontiguousarray(tgt, dtype=np.int64)
    w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
    miss = None if missing is None else np.ascontiguousarray(missing, dtype=np.uint8)
    ne = np.ascontiguousarray(node_ego, dtype=np.int64)
    ee = None if edge_ego is None else np.ascontiguousarray(edge_ego, dtype=np.int64)
    m = len(s)
    off = np.zeros(int(egos) + 1, dtype=np.int64)
    ids = np.zeros(max(int(n), 1), dtype=np.int64)
    rows = np.zeros(max(m, 1), dtype=np.int64)
    cnt = ctypes.c_int64()
    h = ctypes.c_void_p()
    err = ctypes.create_string_buffer(ERR_LEN)
    _check(lib().net_frame_egos(int(n), _ptr(s), _ptr(t), _ptr(w), _ptr(miss), m, int(directed),
                                _ptr(ne), _ptr(ee), int(egos), ctypes.byref(h), _ptr(off),
                                _ptr(ids), _ptr(rows), ctypes.byref(cnt), err, ERR_LEN), err)
    members = int(off[-1])
    g = Graph(members, directed=directed, _handle=h, _m=cnt.value, _weighted=w is not None)
    return g, off, ids[:members], rows[: cnt.value]


def generate_gnm(n, m, directed=False, loops=False, seed=1):
    """G(n[k], m[k]) graphs packed one after another (net_generate_gnm):
    returns (src, tgt) with global node numbers."""
    n = np.ascontiguousarray(np.atleast_1d(n), dtype=np.int64)
    m = np.ascontiguousarray(np.atleast_1d(m), dtype=np.int64)
    tot = int(m.sum())
    src = np.zeros(max(tot, 1), dtype=np.int64)
    tgt = np.zeros(max(tot, 1), dtype=np.int64)
    err = ctypes.create_string_buffer(ERR_LEN)
    _check(lib().net_generate_gnm(len(n), _ptr(n), _ptr(m), int(directed), int(loops), seed,
                                  _ptr(src), _ptr(tgt), err, ERR_LEN), err)
    return src[:tot], tgt[:tot]


def power_law_sizes(count, alpha=2.1, lo=50, hi=50_000, seed=1):
    out = np.zeros(max(count, 1), dtype=np.int64)
    err = ctypes.create_string_buffer(ERR_LEN)
    _check(lib().net_power_law_sizes(count, alpha, lo, hi, seed, _ptr(out), err, ERR_LEN), err)
    return out[:count]


def sweep_timing(phase: int = 1):
    """(launches, total ms, algorithmic bytes per launch) of the merge-path
    sweep kernel in the last PageRank solve of this thread: FP32 sweeps
    (phase 0) or FP64 sweeps (phase 1)."""
    n = ctypes.c_int64()
    ms = ctypes.c_double()
    b = ctypes.c_double()
    lib().net_sweep_timing(phase, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(b))
    return n.value, ms.value, b.value


def set_sweep_timing(on: bool) -> None:
    lib().net_set_sweep_timing(int(on))


TUNE_IPT, TUNE_RELABEL, TUNE_SWITCH_FACTOR, TUNE_SWITCH_FLOOR, TUNE_VARIANT, TUNE_CARVEOUT, \
    TUNE_EGO_THREADS, TUNE_HOT_NODES, TUNE_PERSISTENT, TUNE_REFINE, TUNE_LONG_ROW, \
    TUNE_SMEM_HOT, TUNE_AUTOTUNE, TUNE_BULK_CTAS, TUNE_BULK_SKIP_CHUNK, TUNE_EGO_BIG_NODES, \
    TUNE_EGO_CLUSTER, TUNE_SMALL_EDGES = 0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17
# sweep kernels (TUNE_VARIANT): merge-path warp tiles with L1-filtered
# gathers; the sliced layout at 48 and 64 resident warps per SM, with the
# most gathered values in shared memory, and with the arc streams staged in
# shared memory by bulk copies
VARIANT_WARP_L1, VARIANT_SLICE, VARIANT_SLICE64, VARIANT_SLICE_SMEM, VARIANT_SLICE_BULK = \
    8, 9, 10, 11, 12


def measure_gather(source: int = 0, words: int = 1 << 24) -> float:
    """Random 4-byte gathers per second over the GPU (net_measure_gather):
    source 0 from a device array of `words` FP32 values, 1 from each SM's
    shared memory, 2, 4 or 8 from a cluster's shared memory."""
    r = ctypes.c_double()
    err = ctypes.create_string_buffer(ERR_LEN)
    _check(lib().net_measure_gather(int(source), int(words), ctypes.byref(r), err, ERR_LEN), err)
    return r.value


def set_tuning(key: int, value: float) -> None:
    """Process-wide PageRank tuning (net_set_tuning)."""
    if lib().net_set_tuning(key, float(value)):
        raise EngineError(f"invalid tuning key {key} or value {value}")


def projected_eigen(a):
    """Eigenvalues (ascending) and eigenvectors (columns) of a symmetric
    matrix of order <= 20 by the device solver of the Lanczos process
    (net_projected_eigen)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    vals = np.zeros(n)
    vecs = np.zeros((n, n))
    err = ctypes.create_string_buffer(ERR_LEN)
    _check(lib().net_projected_eigen(n, _ptr(a), _ptr(vals), _ptr(vecs), err, ERR_LEN), err)
    return vals, vecs


def device_sync() -> None:
    err = ctypes.create_string_buffer(ERR_LEN)
    _check(lib().net_device_sync(err, ERR_LEN), err)
