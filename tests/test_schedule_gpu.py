"""The input schedule built on the GPU (snc_b200_inputs_upload) against the
oracle's restatement of build_schedule + run_cpu's per-step injection
(cpu_backend.cpp:43-65, 85-95): per step, the driven input neurons in
ascending id and their amplitudes summed in event order -- bit for bit.

Covers duplicates whose sum depends on the order of addition, channels that
drive several input neurons, dropped events (time, channel or sample out of
range), samples with zero steps, steps holding more entries than one
shared-memory tile (the global-memory merge rounds), and enough steps for a
multi-block scan."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from snc_b200 import _lib
from snc_b200 import runtime as R
from snc_b200.graph import EVENT_DTYPE
from tests.helpers import input_graph as _graph

pytestmark = pytest.mark.gpu


def _read(dg, ev, steps):
    di = R.DeviceInputs(dg, ev, steps)
    TS, B = int(np.sum(steps)), len(steps)
    ptr = np.zeros(TS + B, np.int32)
    nid = np.zeros(max(1, di.entries), np.int32)
    ext = np.zeros(max(1, di.entries), np.float32)
    _lib.check(_lib.lib().snc_b200_inputs_read(di.h, ptr.ctypes.data, nid.ctypes.data,
                                               ext.ctypes.data), "inputs_read")
    return di, ptr, nid[:di.entries], ext[:di.entries]


def _check(g, ev, steps):
    dg = R.DeviceGraph(g)
    di, ptr, nid, ext = _read(dg, ev, steps)
    base = 0
    total = 0
    for b, T in enumerate(steps):
        optr, onid, oext = O.schedule_merged(g, ev, b, int(T))
        p = ptr[base + b: base + b + T + 1]
        assert np.array_equal(p - p[0], optr), f"sample {b}: step pointers"
        got_n, got_e = nid[p[0]:p[-1]], ext[p[0]:p[-1]]
        assert np.array_equal(got_n, onid), f"sample {b}: neurons"
        assert np.array_equal(got_e.view(np.uint32), oext.view(np.uint32)), f"sample {b}: drive bits"
        base += int(T)
        total += onid.shape[0]
    assert di.entries == total
    di.release()
    dg.release()
    return total


def _events(rows):
    ev = np.zeros(len(rows), dtype=EVENT_DTYPE)
    for k, (s, c, t, a) in enumerate(rows):
        ev[k] = (s, c, t, a)
    return ev


def test_order_dependent_duplicates():
    # (1e8 + 1) - 1e8 = 0 but (1e8 - 1e8) + 1 = 1: the sum order shows
    g = _graph(6)
    rows = [(0, 2, 1, 1e8), (0, 2, 1, 1.0), (0, 2, 1, -1e8),
            (0, 4, 1, -1e8), (0, 4, 1, 1e8), (0, 4, 1, 1.0),
            (0, 1, 0, -0.0), (0, 5, 3, 0.25), (0, 0, 3, 0.5), (0, 5, 3, 0.125)]
    assert _check(g, _events(rows), [5]) == 5


def test_fanout_dropped_events_and_zero_step_samples():
    g = _graph(30, fan=3)  # 10 channels of 3 input neurons
    rng = np.random.default_rng(3)
    steps = [7, 0, 12, 1, 0, 9]
    rows = []
    for b, T in enumerate(steps):
        for _ in range(60):
            rows.append((b, int(rng.integers(0, 10)), int(rng.integers(0, max(T, 1))),
                         float(rng.normal())))
    rows += [(0, 10, 1, 1.0), (0, -1, 1, 1.0), (2, 3, 12, 1.0), (2, 3, -1, 1.0),
             (6, 3, 0, 1.0), (-1, 3, 0, 1.0), (1, 2, 0, 5.0)]
    ev = _events(rows)
    ev = ev[rng.permutation(ev.shape[0])]
    _check(g, ev, steps)


@pytest.mark.parametrize("n_ev", [2300, 9000])
def test_steps_larger_than_a_tile(n_ev):
    # one step with more entries than a shared-memory tile (2048): sorted
    # tiles merged in global memory; duplicates straddle the tiles
    g = _graph(5000, seed=1)
    rng = np.random.default_rng(n_ev)
    ch = rng.integers(0, 5000, n_ev)
    ch[: n_ev // 3] = rng.integers(0, 40, n_ev // 3)
    t = np.where(rng.random(n_ev) < 0.99, 2, rng.integers(0, 4, n_ev))
    ev = np.zeros(n_ev, dtype=EVENT_DTYPE)
    ev["channel_id"] = ch
    ev["time"] = t
    ev["amplitude"] = rng.normal(0, 1, n_ev).astype(np.float32) * np.float32(1e3) ** rng.integers(0, 3, n_ev)
    _check(g, ev, [4])


def test_many_steps_multiblock_scan():
    g = _graph(64, seed=2)
    rng = np.random.default_rng(5)
    steps = [300] * 20  # 6000 steps: a two-level scan
    n = 30000
    ev = np.zeros(n, dtype=EVENT_DTYPE)
    ev["sample_id"] = rng.integers(0, 20, n)
    ev["channel_id"] = rng.integers(0, 64, n)
    ev["time"] = rng.integers(0, 300, n)
    ev["amplitude"] = rng.uniform(-1, 1, n).astype(np.float32)
    _check(g, ev, steps)


def test_empty_events():
    g = _graph(8)
    dg = R.DeviceGraph(g)
    di, ptr, nid, ext = _read(dg, np.zeros(0, dtype=EVENT_DTYPE), [4, 0, 2])
    assert di.entries == 0 and not ptr.any()
    di.release()
    dg.release()
