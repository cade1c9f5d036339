"""The device connectome (snc_b200_connectome_*) against the CPU restatement
(oracle/connectome.py, itself pinned to the reference's Connectome):
layered_local, every prune / regrow round (reports, rows, posts, delays,
signed weights, ages) and the device-built graph against the same graph
uploaded from host arrays."""
import numpy as np
import pytest

from oracle import connectome as OC
from snc_b200 import runtime as R
from snc_b200 import structure as ST

pytestmark = pytest.mark.gpu

CASES = [
    ([60, 40, 10], 1500, 5, dict(grow_per_epoch=40)),
    ([50, 30, 30, 6], 1800, 5, dict(grow_per_epoch=60, protect_rounds=1, delay=2, w_grow_init=0.05)),
    ([40, 20, 5], 600, 4, dict(grow_per_epoch=80, locality_window=0.02, protect_rounds=0)),
    ([60, 40, 10], 1500, 4, dict(grow_per_epoch=50, reward_modulated=True, reward_chance=0.2,
                                 reward_floor=0.25)),
    ([800, 300, 10], 24000, 3, dict(grow_per_epoch=300)),
    # a post losing several synapses in one round takes several local picks
    ([30, 12, 4], 900, 4, dict(grow_per_epoch=150, locality_window=0.5, protect_rounds=0)),
]


def same_csr(dev, ref):
    for i, name in enumerate(("row_ptr", "post", "delay", "weight", "age")):
        a, b = np.asarray(dev[i]), np.asarray(ref[i])
        if name == "weight":
            np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32), err_msg=name)
        else:
            np.testing.assert_array_equal(a, b, err_msg=name)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_device_connectome_equals_restatement(case):
    layers, budget, rounds, kw = CASES[case]
    ref = OC.Connectome.layered_local(layers, budget, 1, 0.05, 11 + case)
    dev = ST.DeviceConnectome.layered_local(layers, budget, 1, 0.05, 11 + case)
    same_csr(dev.to_csr(), ref.to_csr())
    rcfg = OC.StructConfig(**kw)
    dcfg = ST.StructConfig(**kw)
    rng = np.random.default_rng(case)
    n = ref.n
    grown = fallback = 0
    for r in range(rounds):
        w = rng.normal(0, 0.3, ref.num_synapses()).astype(np.float32)
        ref.set_edge_weights(w)
        dev.set_edge_weights(w)
        fires = rng.integers(0, 40, n).astype(np.int64)
        fires[rng.random(n) < 0.2] = 0
        reward = float(rng.random())
        rep_r = ref.structural_update(fires, rcfg, reward)
        rep_d = dev.structural_update(fires, dcfg, reward)
        assert rep_d == rep_r, (r, rep_d, rep_r)
        same_csr(dev.to_csr(), ref.to_csr())
        grown += rep_r[1]
        fallback += ref.last_fallback_attempts
    assert grown > 0
    if case == 2:
        assert fallback > 0


def test_device_graph_equals_uploaded_graph():
    """to_graph on the device gives the packed layout and the forward of the
    same graph uploaded from host arrays."""
    layers = [60, 40, 10]
    dev = ST.DeviceConnectome.layered_local(layers, 1500, 1, 0.05, 3)
    rng = np.random.default_rng(0)
    dev.set_edge_weights(rng.normal(0, 0.3, dev.num_synapses()).astype(np.float32))
    dev.structural_update(rng.integers(0, 30, dev.num_neurons), ST.StructConfig(grow_per_epoch=50, delay=3))
    g_dev = dev.to_graph()
    hg = dev.host_graph()
    g_host = R.DeviceGraph(hg)
    from test_graph_layout_gpu import _layout
    (la, bsa, pa), (lb, bsb, pb) = _layout(g_dev, hg), _layout(g_host, hg)
    assert (bsa, pa) == (bsb, pb)
    for k in la:
        np.testing.assert_array_equal(la[k], lb[k], err_msg=k)
    from snc_b200 import workloads as W
    ev, steps = W.random_events(5, dev.host_graph(), 4, [30, 25, 30, 12])
    lif = R.LIFParams(threshold=0.5)
    a = R.forward_batched(g_dev, ev, steps, lif, mode=R.MODE_SORT)
    b = R.forward_batched(g_host, ev, steps, lif, mode=R.MODE_SORT)
    assert int(a["spikes"].sum()) > 0
    for k in ("spikes", "events", "logits"):
        np.testing.assert_array_equal(a[k], b[k])


def test_cotrain_rounds_keep_the_budget():
    """Three co-training rounds on a small layered connectome: e-prop on the
    device graph, weights carried back, prune / regrow between rounds; every
    round's synapse count is the previous one less the pruned plus the
    grown, and the last round's graph has that many synapses."""
    from snc_b200 import eprop as EP
    from snc_b200 import workloads as W
    layers = [40, 24, 4]
    con = ST.DeviceConnectome.layered_local(layers, 960, 1, 0.2, 5)
    S0 = con.num_synapses()
    g = con.host_graph()
    batches = []
    for b in range(2):
        ev, steps = W.random_events(20 + b, g, 8, [25] * 8)
        labels = np.random.default_rng(b).integers(0, 4, 8)
        batches.append((ev, steps, labels))
    cfg = EP.TrainConfig(lr=0.05, lif=R.LIFParams(threshold=0.6), mode=R.MODE_SORT)
    rounds = ST.cotrain(con, batches, cfg, ST.StructConfig(grow_per_epoch=30, protect_rounds=0),
                        outer=3, inner=2, batch=8)
    assert len(rounds) == 3
    assert rounds[0]["pruned"] > 0 and rounds[0]["grown"] > 0
    S = S0
    for r in rounds[:-1]:
        S = S - r["pruned"] + r["grown"]
        assert r["synapses"] == S
    assert con.num_synapses() == S == con.host_graph().num_synapses


def test_prune_at_scale_removes_exactly_the_weakest():
    """Two million synapses, 50 000 pruned: the device removes exactly the K
    smallest (|w|, position) keys (the radix select's eight passes), keeps
    every other edge in its row order with its weight and age advanced,
    appends each grown edge after its pre's kept edges, grows only from the
    previous layer and never duplicates a pair."""
    layers = [20000, 8000, 100]
    dev = ST.DeviceConnectome.layered_local(layers, 2_000_000, 1, 0.05, 9)
    rng = np.random.default_rng(4)
    S = dev.num_synapses()
    w = rng.normal(0, 0.3, S).astype(np.float32)
    w[rng.random(S) < 0.01] = 0.0  # ties of |w| broken by position
    dev.set_edge_weights(w)
    row_ptr, post, delay, w0, age0 = dev.to_csr()
    K = 50_000
    order = np.lexsort((np.arange(S), np.abs(w0)))
    pruned = np.zeros(S, bool)
    pruned[order[:K]] = True
    fires = rng.integers(0, 50, sum(layers)).astype(np.int64)
    rep = dev.structural_update(fires, ST.StructConfig(grow_per_epoch=K, protect_rounds=0, delay=2))
    assert rep[0] == K and 0 < rep[1] <= K and rep[2] == S - K + rep[1]
    rp2, post2, delay2, w2, age2 = dev.to_csr()
    n = sum(layers)
    grown_pairs = set()
    layer_of = np.repeat(np.arange(len(layers)), layers)
    for q in range(n):
        a, b = row_ptr[q], row_ptr[q + 1]
        keep = ~pruned[a:b]
        a2, b2 = rp2[q], rp2[q + 1]
        k = int(keep.sum())
        np.testing.assert_array_equal(post2[a2:a2 + k], post[a:b][keep])
        np.testing.assert_array_equal(w2[a2:a2 + k].view(np.uint32), w0[a:b][keep].view(np.uint32))
        np.testing.assert_array_equal(age2[a2:a2 + k], np.minimum(age0[a:b][keep] + (age0[a:b][keep] < (1 << 20)),
                                                                  1 << 20))
        g = post2[a2 + k:b2]
        assert np.all(delay2[a2 + k:b2] == 2) and np.all(age2[a2 + k:b2] == 1)
        assert len(set(post2[a2:b2].tolist())) == b2 - a2  # no duplicate pair in the row
        for p in g.tolist():
            assert layer_of[p] == layer_of[q] + 1
            grown_pairs.add((q, p))
    assert len(grown_pairs) == rep[1]
