"""The oracle's frame-graph restatement pinned to the reference's own unit
tests of the frame builder (crates/engine/src/frame/build.rs:349-460), with
the tables already resolved to node indices; and the argument checks of the
frame entry points, which run before any device work."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from oracle import oracle as O


def test_unobserved_rows_are_left_out():
    # build.rs:349-385: ids 1..4 resolve to nodes 0..3; rows 1 and 3 are
    # flagged missing.
    src, tgt = [0, 0, 1, 2], [1, 2, 2, 3]
    w = [1.0, 2.0, 3.0, 4.0]
    s, t, ww, rows = O.frame_graph_of(4, src, tgt, w, [False, True, False, True])
    assert s.tolist() == [0, 1] and t.tolist() == [1, 2]
    assert ww.tolist() == [1.0, 3.0] and rows.tolist() == [0, 2]
    # without flags every row is an edge, in row order
    s, t, ww, rows = O.frame_graph_of(4, src, tgt, w, None)
    assert s.tolist() == src and t.tolist() == tgt and rows.tolist() == [0, 1, 2, 3]


def test_ego_subgraphs_of_one_and_two_egos():
    # build.rs:387-425: actors a, b, c of one ego; rows a-b, a-b, b-c, a-a,
    # a-c and an unobserved b-c; edge egos default to the source's.
    src, tgt = [0, 0, 1, 0, 0, 1], [1, 1, 2, 0, 2, 2]
    miss = [False] * 5 + [True]
    w = [1.0, 2.0, 3.0, 4.0, 5.0, 6.0]
    nodes, edges, s, t, ww = O.frame_ego_subgraph(3, src, tgt, w, miss, [0, 0, 0], None, 1, 0)
    assert nodes.tolist() == [0, 1, 2] and edges.tolist() == [0, 1, 2, 3, 4]
    assert ww.tolist() == [1.0, 2.0, 3.0, 4.0, 5.0]
    with pytest.raises(O.OracleError, match="ego index 1 is out of range; the network has 1"):
        O.frame_ego_subgraph(3, src, tgt, w, miss, [0, 0, 0], None, 1, 1)
    # a subgraph without node 1 renumbers the others and drops the rows
    # that touch it (build.rs:429-434)
    nodes, edges, s, t, _ = O.frame_subgraph(3, src, tgt, w, miss, lambda i: i != 1,
                                             lambda e: True)
    assert nodes.tolist() == [0, 2] and edges.tolist() == [3, 4]
    assert s.tolist() == [0, 0] and t.tolist() == [0, 1]
    # two egos p (p, p1) and q (q, q1); rows p-p1, q-q1, q1-q (build.rs:436-452)
    nodes, edges, s, t, ww = O.frame_ego_subgraph(4, [0, 2, 3], [1, 3, 2], None, None,
                                                  [0, 0, 1, 1], None, 2, 1)
    assert nodes.tolist() == [2, 3] and edges.tolist() == [1, 2]
    assert s.tolist() == [0, 1] and ww is None
    with pytest.raises(O.OracleError, match="ego index 2"):
        O.frame_ego_subgraph(4, [0, 2, 3], [1, 3, 2], None, None, [0, 0, 1, 1], None, 2, 2)
    # a frame without an ego role (build.rs:453-459)
    with pytest.raises(O.OracleError, match="no ego role"):
        O.frame_ego_subgraph(2, [0], [1], None, None, None, None, 0, 0)


def test_graph_of_checks_follow_from_edges():
    # graph.rs:162-192: every weight before any endpoint; edges numbered
    # among the observed rows; unobserved rows are never checked.
    src, tgt = [0, 5, 1, 2], [1, 1, 7, 0]
    miss = [False, True, False, False]
    with pytest.raises(O.OracleError,
                       match=r"^edge 1 refers to node index 7, but valid indices are 0\.\.3$"):
        O.frame_graph_of(3, src, tgt, None, miss)
    w = [1.0, 2.0, 3.0, float("nan")]
    with pytest.raises(O.OracleError, match=r"^edge 2 has a missing, NaN, or infinite weight$"):
        O.frame_graph_of(3, src, tgt, w, miss)
    w = [1.0, float("inf"), 3.0, 4.0]
    s, _, _, rows = O.frame_graph_of(8, src, tgt, w, miss)
    assert rows.tolist() == [0, 2, 3] and s.tolist() == [0, 1, 2]


def test_frame_entry_points_check_arguments_before_device_work():
    from knappnet_b200 import build
    build.build()
    import knappnet_b200 as K
    L = K.lib()
    err = ctypes.create_string_buffer(K.ERR_LEN)
    a = np.zeros(4, dtype=np.int64)
    assert L.net_frame_graph(2, K._ptr(a), K._ptr(a), None, None, 4, 1, None, None, None, err,
                             K.ERR_LEN) != 0
    assert b"out is null" in err.value
    h = ctypes.c_void_p()
    assert L.net_frame_graph(2, None, None, None, None, 4, 1, ctypes.byref(h), None, None, err,
                             K.ERR_LEN) != 0
    assert b"endpoint array is null" in err.value
    off = np.zeros(3, dtype=np.int64)
    assert L.net_frame_egos(2, K._ptr(a), K._ptr(a), None, None, 4, 1, K._ptr(a), None, 2,
                            ctypes.byref(h), None, None, None, None, err, K.ERR_LEN) != 0
    assert b"node_offsets is null" in err.value
    assert L.net_frame_egos(2, K._ptr(a), K._ptr(a), None, None, 4, 1, None, None, 2,
                            ctypes.byref(h), K._ptr(off), None, None, None, err, K.ERR_LEN) != 0
    assert b"node_ego is null" in err.value
