"""The Connectome restatement (oracle/connectome.py) pinned to the unchanged
reference (src/structure/connectome.cpp through oracle/ref_shim.cpp) over
several structural rounds: after layered_local and after every prune /
regrow the CSR graphs (rows, posts, delays, signed weights) and the reports
are identical.  Weights are redrawn every round, as training would change
them, so no two eligible synapses tie at the K-th score."""
import numpy as np
import pytest

from oracle import connectome as OC
from oracle import oracle as O

needs_ref = pytest.mark.skipif(not O.ref_available(), reason="reference build (oracle/_ref) absent")


def assert_same(a, b):
    for x, y, name in zip(a[:4], b[:4], ("row_ptr", "post", "delay", "weight")):
        if name == "weight":
            np.testing.assert_array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32))
        else:
            np.testing.assert_array_equal(x, y, err_msg=name)


CASES = [
    # layers, budget, rounds, config
    ([60, 40, 10], 1500, 5, dict(grow_per_epoch=40)),
    ([50, 30, 30, 6], 1800, 5, dict(grow_per_epoch=60, protect_rounds=1, delay=2, w_grow_init=0.05)),
    # narrow windows: most freed posts find no free local pre, so the
    # fallback's random draws are exercised
    ([40, 20, 5], 600, 4, dict(grow_per_epoch=80, locality_window=0.02, protect_rounds=0)),
    ([60, 40, 10], 1500, 4, dict(grow_per_epoch=50, reward_modulated=True, reward_chance=0.2,
                                 reward_floor=0.25)),
]


@needs_ref
@pytest.mark.parametrize("case", range(len(CASES)))
def test_restatement_equals_reference(case):
    layers, budget, rounds, kw = CASES[case]
    ref = OC.RefConnectome(layers, budget, 1, 0.05, 11 + case)
    ours = OC.Connectome.layered_local(layers, budget, 1, 0.05, 11 + case)
    assert_same(ours.to_csr(), ref.to_csr())
    cfg = OC.StructConfig(**kw)
    rng = np.random.default_rng(case)
    n = ours.n
    total_grown = 0
    for r in range(rounds):
        S = ours.num_synapses()
        w = rng.normal(0, 0.3, S).astype(np.float32)
        ours.set_edge_weights(w)
        ref.set_edge_weights(w)
        fires = rng.integers(0, 40, n).astype(np.int64)
        fires[rng.random(n) < 0.2] = 0
        reward = float(rng.random())
        rep_o = ours.structural_update(fires, cfg, reward)
        rep_r = ref.structural_update(fires, cfg, reward)
        assert rep_o == rep_r, (r, rep_o, rep_r)
        assert_same(ours.to_csr(), ref.to_csr())
        total_grown += rep_o[1]
    assert total_grown > 0


def test_fallback_draws_are_reached():
    """The narrow-window case grows through the fallback loop (random posts)
    in its first round: the restatement records the attempts it made."""
    layers, budget, rounds, kw = CASES[2]
    c = OC.Connectome.layered_local(layers, budget, 1, 0.05, 13)
    cfg = OC.StructConfig(**kw)
    rng = np.random.default_rng(2)
    c.set_edge_weights(rng.normal(0, 0.3, c.num_synapses()).astype(np.float32))
    p, g, _ = c.structural_update(rng.integers(0, 40, c.n).astype(np.int64), cfg, 1.0)
    assert p > 0 and g > 0 and c.last_fallback_attempts > 0
