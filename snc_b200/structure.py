"""The co-training loop's structural state on the device.

DeviceConnectome mirrors snc::Connectome (include/snc/connectome.hpp:58-101)
over the C ABI (snc_b200_connectome_*): layered_local, to_graph (a
DeviceGraph built on the device), edge_weights / set_edge_weights,
structural_update and the synapse count.  cotrain() is the reference's
two-timescale loop (src/training/cotrain_main.cpp:247-283) on one GPU:
e-prop rounds on the compiled graph, weights carried back, the firing counts
feeding the prune / regrow step.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import check, lib, ptr
from .graph import INPUT, OUTPUT, SNNGraph
from .runtime import DeviceGraph


@dataclass
class StructConfig:
    """snc::StructConfig (connectome.hpp:33-48), the same defaults."""
    grow_per_epoch: int = 200
    delay: int = 1
    w_grow_init: float = 0.02
    locality_window: float = 0.2
    protect_rounds: int = 2
    max_attempts_mult: int = 8
    reward_modulated: bool = False
    reward_chance: float = 0.1
    reward_floor: float = 0.1

    def c(self):
        return _lib.StructConfig(int(self.grow_per_epoch), int(self.delay), float(self.w_grow_init),
                                 float(self.locality_window), int(self.protect_rounds),
                                 int(self.max_attempts_mult), int(bool(self.reward_modulated)),
                                 float(self.reward_chance), float(self.reward_floor))


class DeviceConnectome:
    def __init__(self, handle, layers):
        self.h = handle
        self.layers = np.ascontiguousarray(layers, np.int32)

    @classmethod
    def layered_local(cls, layers, synapse_budget, delay=1, w_init=0.05, seed=1):
        """Connectome::layered_local (connectome.cpp:14-62)."""
        arr = np.ascontiguousarray(layers, np.int32)
        h = C.c_void_p()
        check(lib().snc_b200_connectome_layered_local(ptr(arr), int(arr.shape[0]), int(synapse_budget),
                                                      int(delay), float(w_init), int(seed), C.byref(h)),
              "connectome_layered_local")
        return cls(h, arr)

    def roles(self):
        """(role, channel) per neuron: the first layer INPUT, the last OUTPUT,
        channel = index within the layer (connectome.cpp:36-39)."""
        n = int(self.layers.sum())
        role = np.zeros(n, np.uint8)
        channel = np.full(n, -1, np.int32)
        L = self.layers.shape[0]
        b = 0
        for li, cnt in enumerate(self.layers):
            if li == 0:
                role[b:b + cnt], channel[b:b + cnt] = INPUT, np.arange(cnt)
            elif li == L - 1:
                role[b:b + cnt], channel[b:b + cnt] = OUTPUT, np.arange(cnt)
            b += cnt
        return role, channel

    def host_graph(self) -> SNNGraph:
        """to_graph() on the host (|weight|, sign +1)."""
        row_ptr, post, delay, w, _ = self.to_csr()
        role, channel = self.roles()
        return SNNGraph(int(self.layers.sum()), row_ptr, post, np.abs(w), delay, role,
                        np.ones(role.shape[0], np.int8), channel)

    def info(self):
        n, s = C.c_int32(), C.c_int32()
        check(lib().snc_b200_connectome_info(self.h, C.byref(n), C.byref(s)), "connectome_info")
        return n.value, s.value

    @property
    def num_neurons(self):
        return self.info()[0]

    def num_synapses(self):
        return self.info()[1]

    def to_csr(self):
        """(row_ptr, post, delay, signed weights, ages) in the reference's
        adjacency order."""
        n, S = self.info()
        row_ptr = np.zeros(n + 1, np.int32)
        post = np.zeros(max(1, S), np.int32)
        delay = np.zeros(max(1, S), np.int32)
        w = np.zeros(max(1, S), np.float32)
        age = np.zeros(max(1, S), np.int32)
        check(lib().snc_b200_connectome_read(self.h, ptr(row_ptr), ptr(post), ptr(delay), ptr(w), ptr(age)),
              "connectome_read")
        return row_ptr, post[:S], delay[:S], w[:S], age[:S]

    def edge_weights(self):
        return self.to_csr()[3]

    def set_edge_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        check(lib().snc_b200_connectome_set_weights(self.h, ptr(w), int(w.shape[0])),
              "connectome_set_weights")

    def structural_update(self, neuron_fires, cfg: StructConfig, reward=1.0):
        """Prune / regrow / age on the device; returns (pruned, grown, synapses)."""
        f = np.ascontiguousarray(neuron_fires, np.int64)
        c = cfg.c()
        r = _lib.StructReport()
        check(lib().snc_b200_connectome_update(self.h, ptr(f), int(f.shape[0]), C.byref(c), float(reward),
                                               C.byref(r)), "connectome_update")
        return r.pruned, r.grown, r.synapses

    def to_graph(self) -> DeviceGraph:
        """to_graph (connectome.cpp:84-101), built on the device."""
        h = C.c_void_p()
        check(lib().snc_b200_connectome_graph(self.h, C.byref(h)), "connectome_graph")
        return DeviceGraph(None, _handle=h)

    def release(self):
        if getattr(self, "h", None):
            lib().snc_b200_connectome_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


def cotrain(con: DeviceConnectome, train, train_cfg, struct_cfg: StructConfig, outer: int,
            inner: int, batch: int):
    """The two-timescale loop of cotrain_main.cpp:247-283 on the device.

    ``train`` is a list of minibatches (events, steps, labels); each outer
    round compiles the connectome (to_graph), runs ``inner`` passes of e-prop
    over the minibatches with the weights carried from the previous round,
    writes the trained weights back, and -- except after the last round --
    prunes and regrows from the round's firing counts with the round's
    training accuracy as the reward.  Returns one dict per round."""
    from .eprop import CudaTrainSession
    rounds = []
    for r in range(outer):
        dg = con.to_graph()
        g = con.host_graph()
        sess = CudaTrainSession(g, train_cfg, batch, weights=con.edge_weights(), device_graph=dg)
        sess.reset_stats()
        correct = total = 0
        for _ in range(inner):
            correct = total = 0
            for ev, steps, labels in train:
                out = sess.run_batch(ev, steps, labels, train=True)
                pred = np.argmax(out["counts"], axis=1)
                correct += int(np.sum(pred == np.asarray(labels)))
                total += len(labels)
        con.set_edge_weights(sess.get_weights())
        _, fires = sess.collect_stats()
        acc = correct / max(1, total)
        rep = (0, 0, con.num_synapses())
        if r < outer - 1 and struct_cfg.grow_per_epoch > 0:
            rep = con.structural_update(fires, struct_cfg, acc)
        rounds.append({"round": r, "train_acc": acc, "pruned": rep[0], "grown": rep[1],
                       "synapses": rep[2]})
        sess.release()
        dg.release()
    return rounds
