"""The CPU oracle (oracle/snc_oracle.c) pinned against the reference.

* golden fixtures written by the UNCHANGED reference (tests/golden) -- always;
* the reference CPU backend itself, compiled from its sources into
  oracle/_ref (skipped where that build is absent): random graphs with
  inhibitory neurons, duplicate synapses and delays, the snc_bench known
  answer, and the reference's own compiler flags (-O3 -march=native) against
  the portable parity build;
* the reference per-sample e-prop Trainer, for the minibatch e-prop
  restatement at batch 1.
"""
import numpy as np
import pytest

from oracle import oracle as O
from snc_b200 import workloads as W
from tests.helpers import golden

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) absent")


@pytest.mark.parametrize("prefix", ["static", "rsparse", "sdelay"])
def test_oracle_matches_reference_fixtures(prefix):
    g, ev, steps, lif, exp = golden(prefix)
    r = O.forward_batched(g, ev, steps, lif)
    np.testing.assert_array_equal(r["spikes"], exp["spikes"])
    np.testing.assert_array_equal(r["events"], exp["events"])
    np.testing.assert_array_equal(r["logits"], exp["logits"])


def test_fixture_sanity():
    g, ev, steps, lif, exp = golden("static")
    assert g.num_neurons == 1050 and g.num_synapses == 40192 and not g.validate()
    assert exp["spikes"].sum() > 0 and exp["events"].sum() > 0


@needs_ref
@pytest.mark.parametrize("seed", [1, 2, 3, 4])
@pytest.mark.parametrize("refractory", [0, 1, 3])
def test_oracle_matches_reference_random(seed, refractory):
    from types import SimpleNamespace
    g = W.random_graph(seed, max_delay=1 + 2 * seed)
    ev, steps = W.random_events(seed + 5, g, 3, 60)
    lif = SimpleNamespace(threshold=1.0, decay=0.9, reset=0.1 * seed, refractory=refractory,
                          reset_mode=0)
    rg = O.RefGraph(g)
    for b in range(3):
        evb = ev[ev["sample_id"] == b]
        r = rg.forward(evb, 60, lif)
        o = O.forward(g, evb, 60, lif)
        assert r["spikes"] == o["spikes"] and r["events"] == o["events"]
        np.testing.assert_array_equal(r["logits"], o["logits"])


@needs_ref
def test_snc_bench_known_answer():
    """snc_bench --structure static-snc --encoder poisson --backend cpu
    --num-steps 50 --num-samples 64 --hidden 256 reports spikes=901715
    synaptic_events=26980240."""
    from types import SimpleNamespace
    g = O.ref_generate("static-snc", [784, 256, 10], synapse_budget=50000, weight=0.5, delay=1,
                       inhib=0.2, seed=1)
    x, _ = O.ref_make_synthetic(64, 784, 10, 0.15, 1)
    lif = SimpleNamespace(threshold=1.0, decay=0.9, reset=0.0, refractory=1, reset_mode=0)
    sp = evn = 0
    for i in range(64):
        ev = O.ref_encode("poisson", x[i], 50, gain=1.0, max_rate=0.5, seed=1 + i)
        o = O.forward(g, ev, 50, lif)
        sp += o["spikes"]
        evn += o["events"]
    assert (sp, evn) == (901715, 26980240)


@needs_ref
def test_reference_flag_sets_agree():
    """The reference's own flags (-O3 -march=native, FMA contraction on)
    give the same outputs as the portable build on the fixtures."""
    if not O.ref_available(native=True):
        pytest.skip("native reference build absent")
    for prefix in ("static", "rsparse", "sdelay"):
        g, ev, steps, lif, exp = golden(prefix)
        rg = O.RefGraph(g, native=True)
        for b in range(len(steps)):
            r = rg.forward(ev[ev["sample_id"] == b], int(steps[b]), lif)
            assert r["spikes"] == exp["spikes"][b] and r["events"] == exp["events"][b]


def test_subtractive_reset_restatement():
    """reset_mode 1 (v -= threshold) has no reference counterpart; with a
    threshold never reached it must equal reset_mode 0 exactly."""
    from types import SimpleNamespace
    g = W.random_graph(3)
    ev, steps = W.random_events(1, g, 2, 40)
    a = O.forward_batched(g, ev, steps, SimpleNamespace(threshold=1e9, decay=0.9, reset=0.0,
                                                      refractory=0, reset_mode=0))
    b = O.forward_batched(g, ev, steps, SimpleNamespace(threshold=1e9, decay=0.9, reset=0.0,
                                                      refractory=0, reset_mode=1))
    np.testing.assert_array_equal(a["v"].view(np.uint32), b["v"].view(np.uint32))
    assert a["spikes"].sum() == 0


def test_batched_equals_per_sample():
    from types import SimpleNamespace
    g = W.random_graph(2)
    ev, steps = W.random_events(2, g, 3, [10, 0, 25])
    lif = SimpleNamespace(threshold=1.0, decay=0.95, reset=0.0, refractory=1, reset_mode=0)
    bt = O.forward_batched(g, ev, steps, lif)
    for b in range(3):
        o = O.forward(g, ev, int(steps[b]), lif, sample=b)
        assert o["spikes"] == bt["spikes"][b]
        np.testing.assert_array_equal(o["v"], bt["v"][b])


@needs_ref
@pytest.mark.parametrize("train_hidden", [False, True])
def test_eprop_restatement_matches_reference_trainer(train_hidden):
    """Minibatch e-prop at batch 1 vs the reference per-sample Trainer
    (src/training/trainer.cpp:154-208).  The Trainer accumulates E in
    double, the minibatch rule in fp32, hence the tolerance."""
    g = O.ref_generate("static-snc", [40, 60, 5], synapse_budget=1500, weight=0.5, delay=2,
                       inhib=0.2, seed=3)
    x, y = O.ref_make_synthetic(1, 40, 5, 0.15, 3)
    cfg = dict(num_steps=30, threshold=1.0, decay=0.9, reset=0.0, refractory=1, encoder="poisson",
               gain=1.0, max_rate=0.5, lr=0.05, w_init=0.3, w_max=4.0, surrogate_scale=0.3,
               feedback_scale=1.0, train_hidden=train_hidden, seed=11)
    ref = O.ref_trainer_one_sample(g, cfg, x[0], int(y[0]), epoch=0)
    from types import SimpleNamespace
    lif = SimpleNamespace(threshold=1.0, decay=0.9, reset=0.0, refractory=1, reset_mode=0)
    ev = ref["events"].copy()
    ev["sample_id"] = 0
    out = O.eprop_batch(g, ref["w_before"], ev, [30], lif, trace_decay=0.9, gamma=0.3, lr=0.05,
                        w_max=4.0, train_hidden=train_hidden, bmat=ref["bmat"], labels=[int(y[0])])
    dw_ref = ref["w_after"] - ref["w_before"]
    dw = out["w"] - ref["w_before"]
    assert np.abs(dw_ref).max() > 0
    np.testing.assert_allclose(dw, dw_ref, rtol=1e-4, atol=1e-6)


def test_schedule_merged_restatement():
    """orc_schedule_merged against a pure-Python statement of the same
    per-step injection: drive summed in event order, neurons ascending."""
    g = W.random_graph(31, n_in=12)
    ev, _ = W.random_events(32, g, 3, [9, 4, 7])
    role, chan = np.asarray(g.role), np.asarray(g.channel)
    nic = int(chan[role == 1].max()) + 1
    members = {c: [i for i in range(g.num_neurons) if role[i] == 1 and chan[i] == c] for c in range(nic)}
    for b, T in enumerate([9, 4, 7]):
        ptr, nid, ext = O.schedule_merged(g, ev, b, T)
        k = 0
        for t in range(T):
            acc = {}
            for e in ev:
                if e["sample_id"] != b or e["time"] != t or not 0 <= e["channel_id"] < nic:
                    continue
                for i in members[int(e["channel_id"])]:
                    acc[i] = np.float32(acc.get(i, np.float32(0.0)) + e["amplitude"])
            assert ptr[t] == k and ptr[t + 1] == k + len(acc)
            for i in sorted(acc):
                assert nid[k] == i and ext[k].view(np.uint32) == np.float32(acc[i]).view(np.uint32)
                k += 1
