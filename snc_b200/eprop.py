"""Minibatch e-prop on the B200: the reference's ``snc::cudatrain`` session
(include/snc/cuda_trainer.hpp:26-57) over the C ABI.

``available / create / destroy / set_weights / get_weights / train_epoch /
evaluate / reset_stats / collect_stats`` keep the reference's names and
meaning.  Differences, by design:
  * inputs are InputEvents encoded on the host (``snc_b200.workloads``'s
    Poisson encoder here; the C++ adapter uses the reference's ``encode``),
    not cuRAND draws, so a minibatch is reproducible and checkable;
  * a minibatch may hold samples of different lengths (lr / T_b per sample);
  * the pre-trace decay is a parameter (the reference ties it to lif.decay);
  * delivery is bit-exact (SORT) by default, ATOMIC on request.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import sys

import numpy as np

from . import _lib
from ._lib import check, lib, ptr
from .graph import INTERNAL, SNNGraph
from .runtime import DeviceGraph, LIFParams, _events


class EpropCfg(C.Structure):
    _fields_ = [("lr", C.c_float), ("w_max", C.c_float), ("surrogate_scale", C.c_float),
                ("trace_decay", C.c_float), ("train_hidden", C.c_int32), ("mode", C.c_int32)]


@dataclasses.dataclass
class TrainConfig:
    """TrainConfig (include/snc/trainer.hpp:30-48) plus trace_decay / mode."""
    num_steps: int = 30
    lif: LIFParams = dataclasses.field(default_factory=LIFParams)
    max_rate: float = 0.5
    gain: float = 1.0
    lr: float = 0.02
    w_init: float = 0.3
    w_max: float = 4.0
    surrogate_scale: float = 0.3
    feedback_scale: float = 1.0
    train_hidden: bool = True
    seed: int = 1
    trace_decay: float | None = None   # None: lif.decay, as the reference
    mode: int = _lib.MODE_SORT


def available(cfg: TrainConfig | None = None) -> bool:
    return bool(lib().snc_b200_available())


class CudaTrainSession:
    """An e-prop session on one device graph.  Weights are signed, in CSR
    order; the feedback matrix has one row per INTERNAL neuron."""

    def __init__(self, g: SNNGraph, cfg: TrainConfig, batch: int, weights=None, feedback=None,
                 device_graph: DeviceGraph | None = None):
        L = lib()
        self.g, self.cfg, self.batch = g, cfg, int(batch)
        self.dg = device_graph or DeviceGraph(g)
        rng = np.random.default_rng(cfg.seed)
        n_int = int((g.role == INTERNAL).sum())
        self.oc = max(1, g.num_output_channels)
        if weights is None:
            weights = rng.uniform(0.0, cfg.w_init, g.num_synapses)
        if feedback is None:
            feedback = rng.normal(0.0, cfg.feedback_scale, (n_int, self.oc))
        w = np.ascontiguousarray(weights, dtype=np.float32)
        fb = np.ascontiguousarray(feedback, dtype=np.float32).reshape(max(1, n_int), self.oc) \
            if n_int else np.zeros((1, self.oc), np.float32)
        self.feedback = fb
        td = cfg.lif.decay if cfg.trace_decay is None else cfg.trace_decay
        self._cfg = EpropCfg(cfg.lr, cfg.w_max, cfg.surrogate_scale, td, int(cfg.train_hidden),
                             int(cfg.mode))
        self._lif = cfg.lif.c()
        h = C.c_void_p()
        check(L.snc_b200_eprop_create(self.dg.h, C.byref(self._lif), C.byref(self._cfg),
                                      self.batch, ptr(w), ptr(fb), C.byref(h)), "eprop_create")
        self.h = h

    # -- cudatrain API ------------------------------------------------------
    def set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        if w.shape[0] != self.g.num_synapses:
            raise ValueError("weights must have one entry per synapse")
        check(lib().snc_b200_eprop_set_weights(self.h, ptr(w)), "eprop_set_weights")

    def uses_grid(self) -> bool:
        """True when the forward runs on the all-SM kernel (one sample's state
        does not fit one CTA's shared memory)."""
        return lib().snc_b200_eprop_path(self.h) == _lib.PATH_PERSISTENT

    def get_weights(self) -> np.ndarray:
        w = np.zeros(self.g.num_synapses, np.float32)
        check(lib().snc_b200_eprop_get_weights(self.h, ptr(w)), "eprop_get_weights")
        return w

    def run_batch(self, events, steps, labels=None, train=True):
        """One minibatch (cuda_trainer.cu run_batch): returns dict(counts
        [B, n_out], spikes, events, ms)."""
        ev = _events(events)
        steps = np.ascontiguousarray(steps, dtype=np.int32)
        B = steps.shape[0]
        lab = None if labels is None else np.ascontiguousarray(labels, dtype=np.int32)
        counts = np.zeros((B, max(1, self.g.num_output_channels)), np.float32)
        st = _lib.RunStats()
        check(lib().snc_b200_eprop_batch(self.h, ptr(ev), ev.shape[0], B, ptr(steps), ptr(lab),
                                         int(bool(train)), ptr(counts), C.byref(st)),
              "eprop_batch")
        return {"counts": counts[:, :self.g.num_output_channels], "spikes": st.spikes,
                "events": st.synaptic_events, "ms": st.ms}

    def gradient(self, events, steps, labels, grad) -> dict:
        """Training minibatch without the update: grad (a float32 CUDA tensor
        [S]) receives sum_b L * E / T_b over these samples."""
        ev = _events(events)
        steps = np.ascontiguousarray(steps, dtype=np.int32)
        lab = np.ascontiguousarray(labels, dtype=np.int32)
        B = steps.shape[0]
        counts = np.zeros((B, max(1, self.g.num_output_channels)), np.float32)
        st = _lib.RunStats()
        check(lib().snc_b200_eprop_gradient(self.h, ptr(ev), ev.shape[0], B, ptr(steps), ptr(lab),
                                            C.c_void_p(grad.data_ptr()), ptr(counts), C.byref(st)),
              "eprop_gradient")
        return {"counts": counts[:, :self.g.num_output_channels], "spikes": st.spikes,
                "events": st.synaptic_events, "ms": st.ms}

    def apply(self, grad, total_batch: int) -> None:
        """w = clamp(w - lr * grad / total_batch) with grad a CUDA tensor [S]."""
        check(lib().snc_b200_eprop_apply(self.h, C.c_void_p(grad.data_ptr()), int(total_batch)),
              "eprop_apply")

    def eligibility(self, B) -> np.ndarray:
        e = np.zeros((B, self.g.num_synapses), np.float32)
        check(lib().snc_b200_eprop_get_eligibility(self.h, ptr(e)), "eprop_get_eligibility")
        return e

    def reset_stats(self):
        check(lib().snc_b200_eprop_reset_stats(self.h), "eprop_reset_stats")

    def collect_stats(self):
        syn = np.zeros(self.g.num_synapses, np.int64)
        neu = np.zeros(self.g.num_neurons, np.int64)
        check(lib().snc_b200_eprop_collect_stats(self.h, ptr(syn), ptr(neu)), "eprop_collect_stats")
        return syn, neu

    def encode(self, X, epoch, indices):
        """Poisson events (rate = feature x max_rate, amplitude = gain) for the
        samples `indices` of X, one seed per (sample, epoch)."""
        from .workloads import poisson_events
        evs = []
        for b, i in enumerate(indices):
            rng = np.random.default_rng([self.cfg.seed, int(i), int(epoch)])
            rates = np.minimum(np.asarray(X[i], np.float32) * np.float32(self.cfg.max_rate), 1.0)
            evs.append(poisson_events(rng, rates, self.cfg.num_steps, sample_id=b,
                                      amplitude=self.cfg.gain))
        return np.concatenate(evs) if evs else None

    def train_epoch(self, X, y, X_test=None, y_test=None, epoch=0) -> dict:
        """One shuffled pass in minibatches (cuda_trainer.cu:392-435)."""
        order = np.random.default_rng([self.cfg.seed, 977, epoch]).permutation(len(X))
        loss, correct, spikes, events = 0.0, 0, 0, 0
        for off in range(0, len(X), self.batch):
            idx = order[off:off + self.batch]
            r = self.run_batch(self.encode(X, epoch, idx), np.full(len(idx), self.cfg.num_steps),
                               np.asarray(y)[idx], train=True)
            c = r["counts"]
            mx = c.max(axis=1, keepdims=True)
            lse = np.log(np.exp(c - mx).sum(axis=1)) + mx[:, 0]
            loss += float((lse - c[np.arange(len(idx)), np.asarray(y)[idx]]).sum())
            correct += int((c.argmax(axis=1) == np.asarray(y)[idx]).sum())
            spikes += r["spikes"]
            events += r["events"]
        out = {"loss": loss / len(X), "train_acc": correct / len(X), "spikes": spikes,
               "synaptic_events": events, "energy": 1.0 * spikes + 0.2 * events}
        out["test_acc"] = self.evaluate(X_test, y_test) if X_test is not None else 0.0
        return out

    def evaluate(self, X, y) -> float:
        correct = 0
        for off in range(0, len(X), self.batch):
            idx = np.arange(off, min(len(X), off + self.batch))
            r = self.run_batch(self.encode(X, 10**6, idx), np.full(len(idx), self.cfg.num_steps),
                               train=False)
            correct += int((r["counts"].argmax(axis=1) == np.asarray(y)[idx]).sum())
        return correct / max(1, len(X))

    def release(self):
        if getattr(self, "h", None):
            lib().snc_b200_eprop_release(self.h)
            self.h = None

    def __del__(self, _finalizing=sys.is_finalizing):
        # a default argument outlives the module globals cleared at exit
        if not _finalizing():  # the library may already be unloaded
            self.release()


def create(g: SNNGraph, cfg: TrainConfig, batch: int, **kw) -> CudaTrainSession:
    return CudaTrainSession(g, cfg, batch, **kw)


def destroy(s: CudaTrainSession) -> None:
    s.release()
