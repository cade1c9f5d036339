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


# ---- SNCG files parsed and packed on the device --------------------------------

def _sncg_bytes(g, tmp_path, with_weights=True):
    from snc_b200.graph import save_sncg
    p = tmp_path / "g.sncg"
    save_sncg(g, p, with_weights=with_weights)
    return p.read_bytes()


@pytest.mark.parametrize("make", [lambda: W.random_graph(3, max_delay=9),
                                  lambda: _many_blocks(1),
                                  lambda: W.rec100k_graph(n=20000, width=200, seed=2)])
@pytest.mark.parametrize("with_weights", [True, False])
def test_sncg_device_ingest_equals_the_host_upload(make, with_weights, tmp_path):
    """The delivery layout built from an SNCG file on the device equals the
    layout of the same graph uploaded from host arrays (weights 1 and signs +1
    when the file has no weights section), and the two uploads share the
    autotuner's content hash."""
    from snc_b200.graph import graph_from_sncg, load_graph
    g = make()
    data = _sncg_bytes(g, tmp_path, with_weights)
    ref_g = graph_from_sncg(load_graph(tmp_path / "g.sncg"))
    dg_file = R.DeviceGraph.from_sncg(data)
    dg_host = R.DeviceGraph(ref_g)
    a, bs_a, p_a = _layout(dg_file, ref_g)
    b, bs_b, p_b = _layout(dg_host, ref_g)
    assert (bs_a, p_a) == (bs_b, p_b)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert (dg_file.N, dg_file.S, dg_file.n_in, dg_file.n_out) == (dg_host.N, dg_host.S, dg_host.n_in,
                                                                   dg_host.n_out)
    # the tuner keys both uploads alike: tuning one is found from the other
    ev, steps = W.random_events(5, ref_g, 1, [20]) if ref_g.num_input_channels else \
        (np.zeros(0, dtype=W.EVENT_DTYPE), [20])
    di_h, di_f = R.DeviceInputs(dg_host, ev, steps), R.DeviceInputs(dg_file, ev, steps)
    if ref_g.num_neurons <= 500:
        R.autotune(dg_host, di_h, R.LIFParams())
        assert R.autotune_lookup(dg_file, di_f) is not None


def test_sncg_device_ingest_forward_and_rejections(tmp_path):
    from oracle import oracle as O
    g = W.random_graph(11, n_hid=80, max_delay=7)
    data = bytearray(_sncg_bytes(g, tmp_path))
    dg = R.DeviceGraph.from_sncg(bytes(data))
    ev, steps = W.random_events(12, g, 2, [30, 25])
    lif = R.LIFParams(refractory=1)
    di = R.DeviceInputs(dg, ev, steps)
    run = R.Run(dg, di, raster=True, vfinal=True)
    run.launch(lif, mode=R.MODE_SORT, path=R.PATH_PERSISTENT)
    out = run.fetch(raster=True, vfinal=True)
    ref = O.forward_batched(g, ev, steps, lif)
    for k in ("spikes", "events", "logits", "raster"):
        assert np.array_equal(out[k], ref[k]), k
    N, S = g.num_neurons, g.num_synapses
    words = np.frombuffer(bytes(data), dtype="<i4").copy()
    # offsets (in words) of pre, post, delays
    o_pre, o_post, o_del = 5, 5 + S, 5 + 2 * S
    cases = []
    bad = words.copy(); bad[o_del + 3] = 0; cases.append((bad, _lib.EINVAL, "delay"))
    bad = words.copy(); bad[o_del + 3] = 300; cases.append((bad, _lib.EUNSUPPORTED, "delay"))
    bad = words.copy(); bad[o_post + 1] = N; cases.append((bad, _lib.EINVAL, "post"))
    bad = words.copy(); bad[o_pre + 2], bad[o_pre + S - 1] = bad[o_pre + S - 1], bad[o_pre + 2]
    cases.append((bad, _lib.EINVAL, "CSR order"))
    for w, code, msg in cases:
        with pytest.raises(_lib.SncB200Error) as ei:
            R.DeviceGraph.from_sncg(w.tobytes())
        assert ei.value.status == code and msg in str(ei.value), (msg, str(ei.value))


# ---- grid graphs generated on the device ----------------------------------------

@pytest.mark.parametrize("kw", [dict(seed=3, width=40, height=30, out_degree=24, long_range=3),
                                dict(seed=9, width=64, height=50, out_degree=40, long_range=5,
                                     sigma=6.0, max_delay=17),
                                dict(seed=5, width=16, height=16, out_degree=8, long_range=0,
                                     max_draws=3)])
def test_device_grid_generator_equals_the_host_statement(kw):
    """snc_b200_graph_generate_grid builds, bit for bit, the graph that
    workloads.grid_graph_host builds from the same spec: the device layout
    equals the statement's layout of the host graph (posts through the ring
    columns, delays, weight bits, groups), and a SORT forward on it equals
    the oracle on the host graph."""
    from oracle import oracle as O
    spec = W.grid_graph_spec(**kw)
    g = W.grid_graph_host(spec)
    assert g.validate() == ""
    dg = R.DeviceGraph.generate_grid(spec)
    assert (dg.N, dg.S) == (g.num_neurons, g.num_synapses)
    got, BS, P = _layout(dg, g)
    exp = _expected(g, BS)
    assert P == exp["P"]
    for k in ("edges", "gedges", "gptr", "groups", "col_of", "colbase", "ibase"):
        assert np.array_equal(got[k], exp[k]), k
    ev, steps = W.rec100k_inputs(g, 2, 60, rate=0.05, seed=kw["seed"])
    lif = W.lif_tau20()
    di = R.DeviceInputs(dg, ev, steps)
    run = R.Run(dg, di, raster=True, vfinal=True)
    run.launch(lif, mode=R.MODE_SORT, path=R.PATH_PERSISTENT)
    out = run.fetch(raster=True, vfinal=True)
    ref = O.forward_batched(g, ev, steps, lif)
    for k in ("spikes", "events", "logits", "raster"):
        assert np.array_equal(out[k], ref[k]), k
