"""The device-built delivery layout of an uploaded graph (packed edges,
destination-grouped edges, groups, inbox and column bases) against a numpy
statement of the same layout: the grouped edges must keep the CSR order
within each destination block, which the bit-exact SORT delivery relies on.
Graphs: duplicate synapses, inhibitory neurons, neurons without synapses,
rows that reach many blocks, and an empty graph."""
import numpy as np
import pytest

from snc_b200 import _lib
from snc_b200 import runtime as R
from snc_b200 import workloads as W
from snc_b200.graph import SNNGraph

pytestmark = pytest.mark.gpu


def _expected(g, BS):
    N, S = g.num_neurons, g.num_synapses
    rp, post = np.asarray(g.row_ptr), np.asarray(g.post_ids)
    indeg = np.bincount(post, minlength=N)
    col_of = np.where(indeg > 0, np.cumsum(indeg > 0) - 1, -1).astype(np.int32)
    pre = np.repeat(np.arange(N), np.diff(rp))
    w = (np.asarray(g.sign, np.float32)[pre] * np.asarray(g.weights, np.float32)).astype(np.float32)
    ex = (col_of[post].astype(np.uint32) | (np.asarray(g.delays).astype(np.uint32) << np.uint32(24)))
    edges = np.stack([ex, w.view(np.uint32)], 1)
    blk = post // BS
    order = np.lexsort((np.arange(S), blk, pre))  # by row, then block, then CSR position
    gedges = edges[order]
    gb = blk[order]
    new_group = np.ones(S, bool)
    new_group[1:] = (pre[order][1:] != pre[order][:-1]) | (gb[1:] != gb[:-1])
    first = np.nonzero(new_group)[0]
    groups = np.stack([gb[first], first], 1).astype(np.int32)
    gptr = np.zeros(N + 1, np.int32)
    np.cumsum(np.bincount(pre[order][first], minlength=N), out=gptr[1:])
    P = max(1, (N + BS - 1) // BS)
    ibase = np.zeros(P + 1, np.int32)
    np.cumsum(np.bincount(groups[:, 0], minlength=P), out=ibase[1:])
    colbase = np.array([np.count_nonzero(col_of[:min(N, b * BS)] >= 0) for b in range(P + 1)], np.int32)
    return dict(edges=edges, gedges=gedges, gptr=gptr, groups=groups, col_of=col_of, colbase=colbase,
                ibase=ibase, P=P)


def _layout(dg, g):
    N, S = g.num_neurons, g.num_synapses
    bs, P, G = (np.zeros(1, np.int32) for _ in range(3))
    L = _lib.lib()
    _lib.check(L.snc_b200_graph_layout(dg.h, *([None] * 7), bs.ctypes.data, P.ctypes.data, G.ctypes.data))
    out = dict(edges=np.zeros((S, 2), np.uint32), gedges=np.zeros((S, 2), np.uint32),
               gptr=np.zeros(N + 1, np.int32), groups=np.zeros((max(1, int(G[0])), 2), np.int32),
               col_of=np.zeros(N, np.int32), colbase=np.zeros(int(P[0]) + 1, np.int32),
               ibase=np.zeros(int(P[0]) + 1, np.int32))
    _lib.check(L.snc_b200_graph_layout(dg.h, *(out[k].ctypes.data for k in
                                               ("edges", "gedges", "gptr", "groups", "col_of",
                                                "colbase", "ibase")), None, None, None))
    out["groups"] = out["groups"][:int(G[0])]
    return out, int(bs[0]), int(P[0])


def _many_blocks(seed):
    # 9000 neurons: 148 blocks; rows spanning many blocks, unsorted posts,
    # repeated (pre, post) pairs with different delays
    rng = np.random.default_rng(seed)
    N = 9000
    deg = rng.integers(0, 400, N)
    deg[::17] = 0
    rp = np.zeros(N + 1, np.int32)
    np.cumsum(deg, out=rp[1:])
    S = int(rp[-1])
    post = rng.integers(0, N, S).astype(np.int32)
    post[1::5] = post[0::5][:post[1::5].shape[0]]
    role = np.zeros(N, np.uint8)
    role[:100] = 1
    role[-10:] = 2
    ch = np.full(N, -1, np.int32)
    ch[:100] = np.arange(100)
    ch[-10:] = np.arange(10)
    sign = np.where(rng.random(N) < 0.2, -1, 1).astype(np.int8)
    return SNNGraph(N, rp, post, rng.normal(0, 0.2, S).astype(np.float32),
                    rng.integers(1, 31, S).astype(np.int32), role, sign, ch)


@pytest.mark.parametrize("make", [lambda: W.random_graph(3, max_delay=9),
                                  lambda: _many_blocks(1),
                                  lambda: W.rec100k_graph(n=20000, width=200, seed=2)])
def test_device_layout_matches_statement(make):
    g = make()
    dg = R.DeviceGraph(g)
    got, BS, P = _layout(dg, g)
    exp = _expected(g, BS)
    assert P == exp["P"]
    for k in ("edges", "gedges", "gptr", "groups", "col_of", "colbase", "ibase"):
        assert np.array_equal(got[k], exp[k]), k
    dg.release()


def test_empty_graph():
    g = SNNGraph(0, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32),
                 np.zeros(0, np.int32), np.zeros(0, np.uint8), np.zeros(0, np.int8),
                 np.zeros(0, np.int32))
    dg = R.DeviceGraph(g)
    got, BS, P = _layout(dg, g)
    assert P == 1 and got["ibase"].tolist() == [0, 0] and got["gptr"].tolist() == [0]
    dg.release()
