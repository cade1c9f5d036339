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


def input_graph(n_in, n_hid=40, fan=1, seed=0):
    """n_in input neurons, `fan` of them per channel (ascending ids), a few
    hidden neurons and one output, sparse random edges."""
    rng = np.random.default_rng(seed)
    N = n_in + n_hid + 1
    pre = rng.integers(0, N - 1, 4 * N)
    post = rng.integers(n_in, N, 4 * N)
    order = np.argsort(pre, kind="stable")
    pre, post = pre[order], post[order]
    row_ptr = np.zeros(N + 1, np.int64)
    np.cumsum(np.bincount(pre, minlength=N), out=row_ptr[1:])
    role = np.zeros(N, np.uint8)
    role[:n_in] = 1
    role[-1] = 2
    channel = np.full(N, -1, np.int32)
    channel[:n_in] = np.arange(n_in) // fan
    channel[-1] = 0
    return SNNGraph(N, row_ptr.astype(np.int32), post.astype(np.int32),
                    rng.uniform(0.1, 0.5, pre.shape[0]).astype(np.float32),
                    rng.integers(1, 5, pre.shape[0]).astype(np.int32), role,
                    np.ones(N, np.int8), channel)
