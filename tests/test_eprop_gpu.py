"""Minibatch e-prop on the GPU against the CPU restatement of the
reference rule (oracle/snc_oracle.c, pinned against the reference Trainer in
tests/test_oracle.py).

With SORT delivery the forward, the surrogate, the traces and the
eligibility are bit-identical to the restatement; the weight update goes
through one softmax whose expf differs between CUDA and glibc by at most a
few ulp, so updated weights are compared with rtol 1e-5.
"""
import numpy as np
import pytest

from oracle import oracle as O
from snc_b200 import eprop as E
from snc_b200 import runtime as R
from snc_b200 import workloads as W
from snc_b200.graph import INTERNAL

pytestmark = pytest.mark.gpu


def make_case(seed, B, steps, n_hid=80, max_delay=6):
    g = W.random_graph(seed, n_hid=n_hid, max_delay=max_delay)
    ev, st = W.random_events(seed + 1, g, B, steps)
    rng = np.random.default_rng(seed)
    w0 = rng.normal(0, 0.5, g.num_synapses).astype(np.float32)
    n_int = int((g.role == INTERNAL).sum())
    fb = rng.normal(0, 1.0, (n_int, g.num_output_channels)).astype(np.float32)
    labels = rng.integers(0, g.num_output_channels, B).astype(np.int32)
    return g, ev, st, w0, fb, labels


@pytest.mark.parametrize("seed,steps,train_hidden", [(1, [40] * 4, True), (2, [30, 55, 10, 44, 5], True),
                                                     (3, [25] * 3, False)])
def test_eprop_matches_restatement(seed, steps, train_hidden):
    B = len(steps)
    g, ev, st, w0, fb, labels = make_case(seed, B, steps)
    lif = R.LIFParams(threshold=1.0, decay=0.9, reset=0.0, refractory=1)
    cfg = E.TrainConfig(lif=lif, lr=0.5, w_max=4.0, surrogate_scale=0.3, train_hidden=train_hidden,
                        trace_decay=0.95)
    s = E.CudaTrainSession(g, cfg, batch=8, weights=w0, feedback=fb)
    fires = np.zeros(g.num_neurons, np.int64)
    ref = O.eprop_batch(g, w0, ev, st, lif, trace_decay=0.95, gamma=0.3, lr=0.5, w_max=4.0,
                        train_hidden=train_hidden, bmat=fb, labels=labels, want_elig=True,
                        fires=fires)
    out = s.run_batch(ev, st, labels, train=True)
    np.testing.assert_array_equal(out["counts"], ref["counts"])
    assert out["spikes"] == ref["spikes"] and out["events"] == ref["events"]
    el = s.eligibility(B)
    np.testing.assert_array_equal(el.view(np.uint32), ref["elig"].view(np.uint32))
    w1 = s.get_weights()
    assert np.abs(w1 - w0).max() > 0
    np.testing.assert_allclose(w1, ref["w"], rtol=1e-5, atol=1e-7)
    syn, neu = s.collect_stats()
    np.testing.assert_array_equal(neu, fires)
    np.testing.assert_array_equal(syn, fires[g.pre_ids()])
    s.reset_stats()
    assert s.collect_stats()[1].sum() == 0


def test_eprop_forward_only_and_weight_roundtrip():
    g, ev, st, w0, fb, labels = make_case(4, 3, [20, 20, 20])
    lif = R.LIFParams(refractory=1)
    s = E.CudaTrainSession(g, E.TrainConfig(lif=lif), batch=4, weights=w0, feedback=fb)
    out = s.run_batch(ev, st, train=False)
    np.testing.assert_array_equal(s.get_weights(), w0)
    ref = O.eprop_batch(g, w0, ev, st, lif, trace_decay=lif.decay, gamma=0.3, lr=0.02, w_max=4.0,
                        train_hidden=True, bmat=fb, labels=labels, train=False)
    np.testing.assert_array_equal(out["counts"], ref["counts"])
    w2 = (w0 * 0.5).astype(np.float32)
    s.set_weights(w2)
    np.testing.assert_array_equal(s.get_weights(), w2)
    assert s.collect_stats()[1].sum() == 0  # evaluation accumulates no statistics


def test_eprop_audio700_minibatch():
    """The batched uneven workload's e-prop update: batch 32 of the 256
    audio700 samples, lr 1.0, trace decay 0.95 (here 8 samples to keep the
    CPU restatement fast)."""
    g = W.audio700_graph()
    ev, st = W.audio700_inputs(8, t_max=300)
    lif = W.lif_tau20()
    rng = np.random.default_rng(5)
    n_int = int((g.role == INTERNAL).sum())
    fb = rng.normal(0, 1.0, (n_int, 20)).astype(np.float32)
    labels = rng.integers(0, 20, 8).astype(np.int32)
    cfg = E.TrainConfig(lif=lif, lr=1.0, trace_decay=0.95, w_max=4.0, surrogate_scale=0.3)
    s = E.CudaTrainSession(g, cfg, batch=32, weights=g.weights, feedback=fb)
    out = s.run_batch(ev, st, labels, train=True)
    ref = O.eprop_batch(g, g.weights, ev, st, lif, trace_decay=0.95, gamma=0.3, lr=1.0, w_max=4.0,
                        train_hidden=True, bmat=fb, labels=labels)
    np.testing.assert_array_equal(out["counts"], ref["counts"])
    np.testing.assert_allclose(s.get_weights(), ref["w"], rtol=1e-5, atol=1e-6)


def test_train_epoch_runs():
    g = W.ff784_graph()
    rng = np.random.default_rng(0)
    X = rng.random((40, 784), dtype=np.float32)
    y = rng.integers(0, 10, 40)
    cfg = E.TrainConfig(lif=W.lif_tau20(), num_steps=20, lr=1.0, max_rate=0.2)
    s = E.create(g, cfg, batch=16, weights=g.weights)
    st = s.train_epoch(X, y, X[:8], y[:8], epoch=0)
    assert st["spikes"] > 0 and 0.0 <= st["test_acc"] <= 1.0
    E.destroy(s)


def test_gradient_shards_and_apply():
    """snc_b200_eprop_gradient over two sample shards, summed, then
    snc_b200_eprop_apply == one minibatch over all samples (data-parallel
    e-prop on one GPU, shards run one after the other)."""
    import torch
    from snc_b200 import parallel as PAR
    g, ev, st, w0, fb, labels = make_case(6, 5, [30, 18, 30, 25, 9])
    lif = R.LIFParams(refractory=1)
    cfg = E.TrainConfig(lif=lif, lr=0.7, w_max=4.0, trace_decay=0.95)
    s = E.CudaTrainSession(g, cfg, batch=8, weights=w0, feedback=fb)
    total = torch.zeros(g.num_synapses, device="cuda")
    for r in range(2):
        e, t, l = PAR.shard_samples(ev, st, labels, r, 2)
        part = torch.zeros(g.num_synapses, device="cuda")
        s.gradient(e, t, l, part)
        total += part
    s.apply(total, 5)
    ref = O.eprop_batch(g, w0, ev, st, lif, trace_decay=0.95, gamma=0.3, lr=0.7, w_max=4.0,
                        train_hidden=True, bmat=fb, labels=labels)
    np.testing.assert_allclose(s.get_weights(), ref["w"], rtol=1e-5, atol=1e-6)
    # the DataParallelEprop wrapper at world size 1 is the same update
    s2 = E.CudaTrainSession(g, cfg, batch=8, weights=w0, feedback=fb)
    PAR.DataParallelEprop(s2, g.num_synapses).step(ev, st, labels)
    np.testing.assert_allclose(s2.get_weights(), ref["w"], rtol=1e-5, atol=1e-6)


@pytest.mark.parametrize("mode", [R.MODE_SORT, R.MODE_ATOMIC])
def test_eprop_on_the_all_sm_path(mode):
    """A sample's state that does not fit one CTA (delays up to 250: a
    251-slot ring) trains on the all-SM kernel: the same eligibility (SORT:
    bit for bit) and update as the restatement, and a second minibatch after
    the update sees the new weights."""
    g = W.random_graph(31, n_hid=300, max_delay=6)
    rng = np.random.default_rng(31)
    d = g.delays.copy()
    d[::3] = rng.integers(100, 251, d[::3].shape[0])
    g.delays = d.astype(np.int32)
    ev, st = W.random_events(32, g, 3, [40, 25, 33])
    w0 = rng.normal(0, 0.5, g.num_synapses).astype(np.float32)
    n_int = int((g.role == INTERNAL).sum())
    fb = rng.normal(0, 1.0, (n_int, g.num_output_channels)).astype(np.float32)
    labels = rng.integers(0, g.num_output_channels, 3).astype(np.int32)
    lif = R.LIFParams(threshold=1.0, decay=0.9, reset=0.0, refractory=1)
    cfg = E.TrainConfig(lif=lif, lr=0.5, w_max=4.0, surrogate_scale=0.3, trace_decay=0.95, mode=mode)
    s = E.CudaTrainSession(g, cfg, batch=4, weights=w0, feedback=fb)
    assert s.uses_grid()
    fires = np.zeros(g.num_neurons, np.int64)
    ref = O.eprop_batch(g, w0, ev, st, lif, trace_decay=0.95, gamma=0.3, lr=0.5, w_max=4.0,
                        train_hidden=True, bmat=fb, labels=labels, want_elig=True, fires=fires)
    out = s.run_batch(ev, st, labels, train=True)
    assert ref["spikes"] > 0
    if mode == R.MODE_SORT:
        np.testing.assert_array_equal(out["counts"], ref["counts"])
        assert out["spikes"] == ref["spikes"] and out["events"] == ref["events"]
        np.testing.assert_array_equal(s.eligibility(3).view(np.uint32), ref["elig"].view(np.uint32))
        np.testing.assert_allclose(s.get_weights(), ref["w"], rtol=1e-5, atol=1e-7)
        np.testing.assert_array_equal(s.collect_stats()[1], fires)
        # second minibatch on the updated weights
        ev2, st2 = W.random_events(33, g, 2, [30, 30])
        lab2 = labels[:2]
        ref2 = O.eprop_batch(g, s.get_weights(), ev2, st2, lif, trace_decay=0.95, gamma=0.3, lr=0.5,
                             w_max=4.0, train_hidden=True, bmat=fb, labels=lab2, train=False)
        out2 = s.run_batch(ev2, st2, train=False)
        np.testing.assert_array_equal(out2["counts"], ref2["counts"])
    else:
        assert abs(out["spikes"] - ref["spikes"]) <= 0.001 * ref["spikes"] + 2


def test_eprop_atomic_small_batch():
    """e-prop with ATOMIC delivery on an audio700 minibatch: the update
    tracks the restatement's -- spike totals within 1 %, the weight change
    correlated above 0.99 (unordered additions move a few spikes)."""
    g = W.audio700_graph()
    ev, st = W.audio700_inputs(8, t_max=300)
    lif = W.lif_tau20()
    rng = np.random.default_rng(5)
    n_int = int((g.role == INTERNAL).sum())
    fb = rng.normal(0, 1.0, (n_int, 20)).astype(np.float32)
    labels = rng.integers(0, 20, 8).astype(np.int32)
    cfg = E.TrainConfig(lif=lif, lr=1.0, trace_decay=0.95, w_max=4.0, surrogate_scale=0.3,
                        mode=R.MODE_ATOMIC)
    w0 = np.asarray(g.weights, np.float32)
    s = E.CudaTrainSession(g, cfg, batch=32, weights=w0, feedback=fb)
    out = s.run_batch(ev, st, labels, train=True)
    ref = O.eprop_batch(g, w0, ev, st, lif, trace_decay=0.95, gamma=0.3, lr=1.0, w_max=4.0,
                        train_hidden=True, bmat=fb, labels=labels)
    assert abs(out["spikes"] - ref["spikes"]) <= 0.01 * ref["spikes"]
    dw, dr = s.get_weights() - w0, ref["w"] - w0
    assert np.abs(dr).max() > 0
    assert float(np.corrcoef(dw, dr)[0, 1]) > 0.99
