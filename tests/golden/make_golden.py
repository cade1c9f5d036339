"""Writes tests/golden/golden_ref.npz from the UNCHANGED reference.

Run where the reference tree is present (it builds oracle/_ref with
`make -C oracle ref`):

    python tests/golden/make_golden.py

Every number in the fixture comes from the reference's own code, called
through oracle/ref_shim.cpp: graphs from snc::make_static_snc /
snc::make_random_sparse (as snc_bench builds them, src/bench/snc_bench.cpp:
123-134), inputs from snc::make_synthetic + snc::encode with the bench's
per-sample seeds (snc_bench.cpp:196-198), outputs from snc::forward with the
serial cpu backend.  The reference's own tests hold no golden vectors for
this path, so these fixtures are the pin.
"""
from __future__ import annotations

import os
import subprocess
import sys
from types import SimpleNamespace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402


def graph_arrays(prefix, g):
    return {f"{prefix}_row_ptr": g.row_ptr, f"{prefix}_post": g.post_ids, f"{prefix}_w": g.weights,
            f"{prefix}_delays": g.delays, f"{prefix}_role": g.role, f"{prefix}_sign": g.sign,
            f"{prefix}_channel": g.channel}


def case(prefix, structure, layers, budget, delay, inhib, seed, steps, samples, decay, refractory,
         max_rate=0.5, native=False):
    g = O.ref_generate(structure, layers, synapse_budget=budget, weight=0.5, delay=delay,
                       inhib=inhib, seed=seed, native=native)
    x, y = O.ref_make_synthetic(samples, layers[0], layers[-1], 0.15, seed, native=native)
    lif = SimpleNamespace(threshold=1.0, decay=decay, reset=0.0, refractory=refractory, reset_mode=0)
    rg = O.RefGraph(g, native=native)
    evs, logits, spikes, events = [], [], [], []
    for i in range(samples):
        ev = O.ref_encode("poisson", x[i], steps, gain=1.0, max_rate=max_rate, seed=seed + i,
                          sample_id=i, native=native)
        r = rg.forward(ev, steps, lif)
        evs.append(ev)
        logits.append(r["logits"])
        spikes.append(r["spikes"])
        events.append(r["events"])
    out = graph_arrays(prefix, g)
    ev = np.concatenate(evs)
    out.update({f"{prefix}_events": ev.view(np.int32).reshape(-1, 4),
                f"{prefix}_steps": np.full(samples, steps, np.int32),
                f"{prefix}_lif": np.array([1.0, decay, 0.0, refractory], np.float32),
                f"{prefix}_logits": np.stack(logits), f"{prefix}_spikes": np.array(spikes),
                f"{prefix}_nevents": np.array(events)})
    return out


def main():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"])
    out = {}
    # snc_bench --structure static-snc --encoder poisson --backend cpu
    #           --num-steps 50 --num-samples 64 --hidden 256 (first 8 samples)
    out.update(case("static", "static-snc", [784, 256, 10], 50000, 1, 0.2, 1, 50, 8, 0.9, 1))
    # random-sparse, inhibitory half, decay 0.95, delay 3
    out.update(case("rsparse", "random-sparse", [100, 200, 10], 6000, 3, 0.5, 7, 80, 6, 0.95, 1))
    # static-snc with delay 4 and refractory 2
    out.update(case("sdelay", "static-snc", [64, 128, 8], 3000, 4, 0.3, 3, 60, 6, 0.9, 2,
                    max_rate=0.8))
    np.savez_compressed(os.path.join(HERE, "golden_ref.npz"), **out)
    print("wrote", os.path.join(HERE, "golden_ref.npz"), {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
