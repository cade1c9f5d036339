"""Shared helpers for the tests."""
from __future__ import annotations

import os
from types import SimpleNamespace

import numpy as np

from snc_b200.graph import EVENT_DTYPE, SNNGraph

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_ref.npz")
_CACHE = {}


def golden(prefix):
    """(graph, events, steps, lif, expected) of one reference fixture case."""
    if "z" not in _CACHE:
        _CACHE["z"] = dict(np.load(GOLDEN))
    z = _CACHE["z"]
    g = SNNGraph(int(z[f"{prefix}_role"].shape[0]), z[f"{prefix}_row_ptr"], z[f"{prefix}_post"],
                 z[f"{prefix}_w"], z[f"{prefix}_delays"], z[f"{prefix}_role"], z[f"{prefix}_sign"],
                 z[f"{prefix}_channel"])
    ev = np.ascontiguousarray(z[f"{prefix}_events"]).view(EVENT_DTYPE).reshape(-1)
    lv = z[f"{prefix}_lif"]
    lif = SimpleNamespace(threshold=float(lv[0]), decay=float(lv[1]), reset=float(lv[2]),
                          refractory=int(lv[3]), reset_mode=0)
    exp = {"logits": z[f"{prefix}_logits"], "spikes": z[f"{prefix}_spikes"],
           "events": z[f"{prefix}_nevents"]}
    return g, ev, z[f"{prefix}_steps"], lif, exp


def to_lif(ns):
    from snc_b200.runtime import LIFParams
    return LIFParams(ns.threshold, ns.decay, ns.reset, ns.refractory, ns.reset_mode)


def spike_count_agreement(a, b):
    """min/max of total spike counts (1.0 when identical)."""
    a, b = float(np.sum(a)), float(np.sum(b))
    if max(a, b) == 0:
        return 1.0
    return min(a, b) / max(a, b)
