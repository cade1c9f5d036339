"""ctypes bindings for the CPU checkers (TEST INFRASTRUCTURE ONLY).

Loaded only by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
reference legs.  Two libraries:

* ``liboracle.so`` -- snc_oracle.c, our C restatement of the reference hot
  path (forward, batched forward, minibatch e-prop).  Always available: it is
  rebuilt from source with gcc when missing.
* ``_ref/libsncref.so`` -- the UNCHANGED reference CPU sources plus
  ref_shim.cpp, built by ``make -C oracle ref`` where the reference tree is
  present.  Used to pin the restatement and as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from snc_b200.graph import EVENT_DTYPE, SNNGraph

HERE = os.path.dirname(os.path.abspath(__file__))
_ORC = None
_REF = {}


class _Graph(C.Structure):
    _fields_ = [("num_neurons", C.c_int32), ("num_synapses", C.c_int32),
                ("row_ptr", C.c_void_p), ("post_ids", C.c_void_p), ("weights", C.c_void_p),
                ("delays", C.c_void_p), ("role", C.c_void_p), ("sign", C.c_void_p),
                ("channel", C.c_void_p)]


class _Lif(C.Structure):
    _fields_ = [("threshold", C.c_float), ("decay", C.c_float), ("reset", C.c_float),
                ("refractory", C.c_int32), ("reset_mode", C.c_int32)]


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def lib():
    """The restatement library, built with gcc on first use if absent."""
    global _ORC
    if _ORC is None:
        path = os.path.join(HERE, "liboracle.so")
        src = os.path.join(HERE, "snc_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", HERE, "all"])
        _ORC = C.CDLL(path)
        for name in ("orc_forward", "orc_forward_batched", "orc_eprop_batch",
                     "orc_ring_len", "orc_num_output_channels"):
            getattr(_ORC, name).restype = C.c_int
    return _ORC


def graph_struct(g: SNNGraph):
    s = _Graph(g.num_neurons, g.num_synapses, _ptr(g.row_ptr), _ptr(g.post_ids),
               _ptr(g.weights), _ptr(g.delays), _ptr(g.role), _ptr(g.sign), _ptr(g.channel))
    return s


def lif_struct(lif):
    return _Lif(lif.threshold, lif.decay, lif.reset, lif.refractory, lif.reset_mode)


def forward(g: SNNGraph, events, num_steps, lif, sample=-1):
    """One sample of the reference's serial run_cpu (cpu_backend.cpp:67-191).
    Returns dict(logits, spikes, events, raster [T, ceil(N/32)] uint32, v)."""
    events = np.ascontiguousarray(events, dtype=EVENT_DTYPE)
    gs = graph_struct(g)
    lf = lif_struct(lif)
    W = (g.num_neurons + 31) // 32
    logits = np.zeros(max(1, g.num_output_channels), np.float32)
    raster = np.zeros((max(num_steps, 0), W), np.uint32)
    v = np.zeros(g.num_neurons, np.float32)
    sp, ev = C.c_int64(), C.c_int64()
    rc = lib().orc_forward(C.byref(gs), _ptr(events), C.c_size_t(events.shape[0]), sample,
                           num_steps, C.byref(lf), _ptr(logits), C.byref(sp), C.byref(ev),
                           _ptr(raster), _ptr(v))
    if rc:
        raise RuntimeError(f"orc_forward failed: {rc}")
    return {"logits": logits[:g.num_output_channels], "spikes": sp.value, "events": ev.value,
            "raster": raster, "v": v}


def forward_batched(g: SNNGraph, events, steps, lif, ro_decay=None):
    """Per-sample run_cpu with per-sample step counts; events carry sample_id.
    ro_decay: OUTPUT neurons with a channel are leaky readout units (logits =
    their final potential / T)."""
    events = np.ascontiguousarray(events, dtype=EVENT_DTYPE)
    steps = np.ascontiguousarray(steps, dtype=np.int32)
    B = steps.shape[0]
    gs, lf = graph_struct(g), lif_struct(lif)
    W = (g.num_neurons + 31) // 32
    oc = max(1, g.num_output_channels)
    logits = np.zeros((B, oc), np.float32)
    spikes = np.zeros(B, np.int64)
    evs = np.zeros(B, np.int64)
    raster = np.zeros((int(steps.sum()), W), np.uint32)
    v = np.zeros((B, g.num_neurons), np.float32)
    f = lib().orc_forward_batched_ro
    f.argtypes = None
    rc = f(C.byref(gs), _ptr(events), C.c_size_t(events.shape[0]), B, _ptr(steps), C.byref(lf),
           C.c_float(-1.0 if ro_decay is None else float(ro_decay)), _ptr(logits), _ptr(spikes),
           _ptr(evs), _ptr(raster), _ptr(v))
    if rc:
        raise RuntimeError(f"orc_forward_batched failed: {rc}")
    return {"logits": logits[:, :g.num_output_channels], "spikes": spikes, "events": evs,
            "raster": raster, "v": v}


def schedule_merged(g: SNNGraph, events, sample: int, T: int):
    """Per step, the driven input neurons (ascending) and their drive summed in
    event order.  Returns (step_ptr [T+1], nid [E], ext [E])."""
    events = np.ascontiguousarray(events, dtype=EVENT_DTYPE)
    gs = graph_struct(g)
    cap = max(1, int(events.shape[0]) * max(1, int(np.bincount(
        np.asarray(g.channel)[np.asarray(g.role) == 1]).max()) if (np.asarray(g.role) == 1).any() else 1))
    ptr = np.zeros(T + 1, np.int32)
    nid = np.zeros(cap, np.int32)
    ext = np.zeros(cap, np.float32)
    f = lib().orc_schedule_merged
    f.restype = C.c_longlong
    n = f(C.byref(gs), _ptr(events), C.c_size_t(events.shape[0]), int(sample), int(T), _ptr(ptr),
          _ptr(nid), _ptr(ext), C.c_longlong(cap))
    if n < 0:
        raise RuntimeError("orc_schedule_merged: capacity")
    return ptr, nid[:n].copy(), ext[:n].copy()


def eprop_batch(g: SNNGraph, w, events, steps, lif, *, trace_decay, gamma, lr, w_max,
                train_hidden, bmat, labels, train=True, want_elig=False, fires=None,
                want_grad=False):
    """Minibatch e-prop restatement (cuda_trainer.cu rule, host events).
    Returns dict(w (updated copy), counts [B, oc], elig [B, S] or None,
    grad [S] or None (want_grad: the shard gradient, w unchanged), spikes,
    events)."""
    events = np.ascontiguousarray(events, dtype=EVENT_DTYPE)
    steps = np.ascontiguousarray(steps, dtype=np.int32)
    B = steps.shape[0]
    w = np.array(w, dtype=np.float32, copy=True)
    gs, lf = graph_struct(g), lif_struct(lif)
    oc = max(1, g.num_output_channels)
    counts = np.zeros((B, oc), np.float32)
    elig = np.zeros((B, g.num_synapses), np.float32) if want_elig else None
    bmat = np.ascontiguousarray(bmat, dtype=np.float32)
    labels = np.ascontiguousarray(labels, dtype=np.int32)
    grad = np.zeros(g.num_synapses, np.float32) if want_grad else None
    sp, ev = C.c_int64(), C.c_int64()
    rc = lib().orc_eprop_batch(C.byref(gs), _ptr(w), _ptr(events), C.c_size_t(events.shape[0]),
                               B, _ptr(steps), C.byref(lf), C.c_float(trace_decay),
                               C.c_float(gamma), C.c_float(lr), C.c_float(w_max),
                               int(bool(train_hidden)), _ptr(bmat), _ptr(labels),
                               int(bool(train)), _ptr(counts), _ptr(elig), C.byref(sp),
                               C.byref(ev), _ptr(fires), _ptr(grad))
    if rc:
        raise RuntimeError(f"orc_eprop_batch failed: {rc}")
    return {"w": w, "counts": counts, "elig": elig, "grad": grad, "spikes": sp.value,
            "events": ev.value}


# ---------------------------------------------------------------------------
# The unchanged reference, through ref_shim.cpp
# ---------------------------------------------------------------------------

def ref_path(native=False):
    return os.path.join(HERE, "_ref", "libsncref_native.so" if native else "libsncref.so")


def ref_available(native=False) -> bool:
    return os.path.exists(ref_path(native))


def ref_lib(native=False):
    if native not in _REF:
        L = C.CDLL(ref_path(native))
        L.ref_graph_create.restype = C.c_void_p
        L.ref_graph_create.argtypes = [C.c_int, C.c_int] + [C.c_void_p] * 7
        L.ref_graph_destroy.argtypes = [C.c_void_p]
        L.ref_graph_validate.argtypes = [C.c_void_p, C.c_char_p, C.c_int]
        L.ref_forward.restype = C.c_double
        L.ref_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_float, C.c_float,
                                  C.c_float, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_encode.restype = C.c_int64
        L.ref_encode.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float,
                                 C.c_float, C.c_uint64, C.c_int, C.c_void_p, C.c_int64]
        L.ref_generate.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int,
                                   C.c_float, C.c_uint64, C.c_void_p, C.c_void_p]
        L.ref_last_graph.argtypes = [C.c_void_p] * 7
        L.ref_make_synthetic.argtypes = [C.c_int, C.c_int, C.c_int, C.c_float, C.c_uint64,
                                         C.c_void_p, C.c_void_p]
        L.ref_trainer_one_sample.restype = C.c_int64
        L.ref_trainer_one_sample.argtypes = (
            [C.c_void_p, C.c_int, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int, C.c_float,
             C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int,
             C.c_uint64, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
             C.c_void_p, C.c_int64])
        _REF[native] = L
    return _REF[native]


class RefGraph:
    """An snc::SNNGraph owned by the reference library."""

    def __init__(self, g: SNNGraph, native=False):
        self.g, self.L = g, ref_lib(native)
        self.h = self.L.ref_graph_create(g.num_neurons, g.num_synapses, _ptr(g.row_ptr),
                                         _ptr(g.post_ids), _ptr(g.weights), _ptr(g.delays),
                                         _ptr(g.role), _ptr(g.sign), _ptr(g.channel))

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_graph_destroy(self.h)
            self.h = None

    def forward(self, events, num_steps, lif, backend="cpu"):
        """snc::forward through the reference; returns dict(logits, spikes,
        events, ms) with ms = the reference's RunStats.ms."""
        events = np.ascontiguousarray(events, dtype=EVENT_DTYPE)
        logits = np.zeros(max(1, self.g.num_output_channels), np.float32)
        sp, ev = C.c_int64(), C.c_int64()
        ms = self.L.ref_forward(self.h, _ptr(events), events.shape[0], num_steps,
                                lif.threshold, lif.decay, lif.reset, lif.refractory,
                                1 if backend == "openmp" else 0, _ptr(logits),
                                C.byref(sp), C.byref(ev))
        return {"logits": logits[:self.g.num_output_channels], "spikes": sp.value,
                "events": ev.value, "ms": ms}


ENCODERS = {"direct": 0, "poisson": 1, "latency": 2}


def ref_encode(encoder, features, num_steps, gain=1.0, max_rate=0.5, threshold=0.0, seed=1,
               sample_id=0, native=False):
    """snc::encode (encoders.cpp:25-71) through the reference library."""
    L = ref_lib(native)
    f = np.ascontiguousarray(features, dtype=np.float32)
    n = L.ref_encode(ENCODERS[encoder], _ptr(f), f.shape[0], num_steps, gain, max_rate,
                     threshold, seed, sample_id, None, 0)
    out = np.zeros(n, dtype=EVENT_DTYPE)
    L.ref_encode(ENCODERS[encoder], _ptr(f), f.shape[0], num_steps, gain, max_rate, threshold,
                 seed, sample_id, _ptr(out), n)
    return out


STRUCTURES = {"dense": 0, "random-sparse": 1, "static-snc": 2}


def ref_generate(structure, layers, synapse_budget=50000, weight=0.5, delay=1, inhib=0.2,
                 seed=1, native=False) -> SNNGraph:
    """The reference generators as snc_bench builds them (snc_bench.cpp:123-134)."""
    L = ref_lib(native)
    lay = np.ascontiguousarray(layers, dtype=np.int32)
    n, s = C.c_int(), C.c_int()
    L.ref_generate(STRUCTURES[structure], _ptr(lay), lay.shape[0], synapse_budget, weight, delay,
                   inhib, seed, C.byref(n), C.byref(s))
    N, S = n.value, s.value
    a = dict(row_ptr=np.zeros(N + 1, np.int32), post=np.zeros(S, np.int32),
             w=np.zeros(S, np.float32), d=np.zeros(S, np.int32), role=np.zeros(N, np.uint8),
             sign=np.zeros(N, np.int8), ch=np.zeros(N, np.int32))
    L.ref_last_graph(*(_ptr(a[k]) for k in ("row_ptr", "post", "w", "d", "role", "sign", "ch")))
    return SNNGraph(N, a["row_ptr"], a["post"], a["w"], a["d"], a["role"], a["sign"], a["ch"])


def ref_make_synthetic(n, dim, classes, noise, seed, native=False):
    L = ref_lib(native)
    x = np.zeros((n, dim), np.float32)
    y = np.zeros(n, np.int32)
    L.ref_make_synthetic(n, dim, classes, noise, seed, _ptr(x), _ptr(y))
    return x, y


def ref_trainer_one_sample(g: SNNGraph, cfg: dict, x, label, epoch=0, native=False):
    """One reference Trainer epoch on a one-sample dataset.  Returns dict(
    w_before, w_after, bmat, events)."""
    rg = RefGraph(g, native)
    L = rg.L
    S = g.num_synapses
    n_internal = int((g.role == 0).sum())
    classes = max(1, g.num_output_channels)
    w0 = np.zeros(S, np.float32)
    w1 = np.zeros(S, np.float32)
    bmat = np.zeros(n_internal * classes, np.float32)
    cap = 1 << 22
    ev = np.zeros(cap, dtype=EVENT_DTYPE)
    xf = np.ascontiguousarray(x, dtype=np.float32)
    n = L.ref_trainer_one_sample(
        rg.h, cfg["num_steps"], cfg["threshold"], cfg["decay"], cfg["reset"], cfg["refractory"],
        ENCODERS[cfg["encoder"]], cfg["gain"], cfg["max_rate"], cfg["lr"], cfg["w_init"],
        cfg["w_max"], cfg["surrogate_scale"], cfg["feedback_scale"], int(cfg["train_hidden"]),
        cfg["seed"], _ptr(xf), int(label), int(epoch), _ptr(w0), _ptr(w1), _ptr(bmat),
        _ptr(ev), cap)
    return {"w_before": w0, "w_after": w1, "bmat": bmat.reshape(n_internal, classes),
            "events": ev[:n].copy()}
