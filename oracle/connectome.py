"""CPU restatement of the reference's Connectome (test infrastructure only).

The co-training loop's structural state: a layered, position-aware edge list
with per-edge ages, compiled to a CSR graph for training, and its prune /
regrow step.  Restated from
  src/structure/connectome.cpp:9-11     layer_pos
  src/structure/connectome.cpp:14-62    Connectome::layered_local
  src/structure/connectome.cpp:70-101   connected, to_graph
  src/structure/connectome.cpp:103-119  edge_weights / set_edge_weights
  src/structure/connectome.cpp:121-219  Connectome::structural_update
with every float expression rounded as the reference's float arithmetic
rounds it.  Random draws come from the C++ library's mt19937_64 and
distributions (oracle/stdrng.cpp), the ones the reference calls.

One choice is the restatement's: the K weakest eligible synapses are the K
smallest by (|weight|, pre, position in the pre's list).  The reference
selects them with std::nth_element, which leaves the choice among equal
scores at the K-th place to the library; where the K-th smallest score is
unique both choose the same set.

Pinned against the unchanged reference (oracle/ref_shim.cpp, ref_con_*) over
several structural rounds in tests/test_connectome.py.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
f32 = np.float32
AGE_CAP = 1 << 20
_RNG = None


def _rng_lib():
    global _RNG
    if _RNG is None:
        path = os.path.join(HERE, "libstdrng.so")
        src = os.path.join(HERE, "stdrng.cpp")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", HERE, "all"])
        L = C.CDLL(path)
        L.srng_new.restype = C.c_void_p
        L.srng_new.argtypes = [C.c_uint64]
        L.srng_copy.restype = C.c_void_p
        L.srng_copy.argtypes = [C.c_void_p]
        L.srng_free.argtypes = [C.c_void_p]
        L.srng_uniform_float.restype = C.c_float
        L.srng_uniform_float.argtypes = [C.c_void_p, C.c_float, C.c_float]
        L.srng_uniform_int.restype = C.c_int
        L.srng_uniform_int.argtypes = [C.c_void_p, C.c_int, C.c_int]
        _RNG = L
    return _RNG


class StdRng:
    """std::mt19937_64 with the library's distributions."""

    def __init__(self, seed):
        self.h = _rng_lib().srng_new(int(seed) & 0xFFFFFFFFFFFFFFFF)

    def uniform_float(self, a, b):
        return f32(_rng_lib().srng_uniform_float(self.h, float(a), float(b)))

    def uniform_int(self, a, b):
        return int(_rng_lib().srng_uniform_int(self.h, int(a), int(b)))

    def __del__(self):
        if getattr(self, "h", None):
            _rng_lib().srng_free(self.h)
            self.h = None


def lround(x) -> int:
    """C lround: nearest integer, halves away from zero."""
    x = float(x)
    return int(math.copysign(math.floor(abs(x) + 0.5), x))


def layer_pos(k, cnt):
    return f32(f32(k) / f32(cnt - 1)) if cnt > 1 else f32(0.5)


class StructConfig:
    """include/snc/connectome.hpp:33-48 (defaults included)."""

    def __init__(self, grow_per_epoch=200, delay=1, w_grow_init=0.02, locality_window=0.2,
                 protect_rounds=2, max_attempts_mult=8, reward_modulated=False, reward_chance=0.1,
                 reward_floor=0.1):
        self.grow_per_epoch, self.delay = int(grow_per_epoch), int(delay)
        self.w_grow_init, self.locality_window = f32(w_grow_init), f32(locality_window)
        self.protect_rounds, self.max_attempts_mult = int(protect_rounds), int(max_attempts_mult)
        self.reward_modulated = bool(reward_modulated)
        self.reward_chance, self.reward_floor = f32(reward_chance), f32(reward_floor)


class Connectome:
    def __init__(self):
        self.n = 0
        self.layer, self.pos, self.role, self.channel = [], [], [], []
        self.layer_begin, self.layer_count = [], []
        self.adj = []  # per pre: list of [post, delay, weight (f32, signed), age]
        self.rng = None

    @staticmethod
    def layered_local(layers, synapse_budget, delay, w_init, seed):
        """connectome.cpp:14-62."""
        c = Connectome()
        L = len(layers)
        c.n = int(sum(layers))
        c.layer, c.pos = [0] * c.n, [f32(0)] * c.n
        c.role, c.channel = [0] * c.n, [-1] * c.n
        c.adj = [[] for _ in range(c.n)]
        c.layer_begin, c.layer_count = [0] * L, [0] * L
        c.rng = StdRng(seed)
        idx = 0
        for li in range(L):
            c.layer_begin[li], c.layer_count[li] = idx, int(layers[li])
            for k in range(layers[li]):
                c.layer[idx] = li
                c.pos[idx] = layer_pos(k, layers[li])
                if li == 0:
                    c.role[idx], c.channel[idx] = 1, k
                elif li == L - 1:
                    c.role[idx], c.channel[idx] = 2, k
                idx += 1
        forward_pre = sum(layers[:-1]) if L > 1 else 0
        fanout = max(1, int(synapse_budget // forward_pre)) if forward_pre > 0 else 0
        for li in range(L - 1):
            from0, from_n = c.layer_begin[li], c.layer_count[li]
            to0, to_n = c.layer_begin[li + 1], c.layer_count[li + 1]
            k = min(fanout, to_n)
            for a in range(from_n):
                j = c.rng.uniform_float(-0.5, 0.5)
                pa = f32(layer_pos(a, from_n) + f32(j / f32(max(1, to_n))))
                centre = lround(f32(pa * f32(to_n - 1)))
                centre = min(max(centre, 0), max(0, to_n - 1))
                lo = min(max(centre - k // 2, 0), max(0, to_n - k))
                for jj in range(k):
                    c.adj[from0 + a].append([to0 + lo + jj, int(delay), f32(w_init), AGE_CAP])
        return c

    def num_synapses(self):
        return sum(len(a) for a in self.adj)

    def connected(self, pre, post):
        return any(e[0] == post for e in self.adj[pre])

    def to_csr(self):
        """to_graph()'s CSR (row_ptr, post, delay) and edge_weights() (signed)."""
        row_ptr = np.zeros(self.n + 1, np.int32)
        for i in range(self.n):
            row_ptr[i + 1] = row_ptr[i] + len(self.adj[i])
        post = np.array([e[0] for a in self.adj for e in a], np.int32)
        delay = np.array([e[1] for a in self.adj for e in a], np.int32)
        w = np.array([e[2] for a in self.adj for e in a], np.float32)
        age = np.array([e[3] for a in self.adj for e in a], np.int32)
        return row_ptr, post, delay, w, age

    def set_edge_weights(self, w):
        idx = 0
        for a in self.adj:
            for e in a:
                if idx >= len(w):
                    return
                e[2] = f32(w[idx])
                idx += 1

    def grow_target(self, cfg, reward):
        g = cfg.grow_per_epoch
        if cfg.reward_modulated:
            denom = max(f32(1e-3), f32(f32(1.0) - cfg.reward_chance))
            comp = min(max(f32(f32(f32(reward) - cfg.reward_chance) / denom), f32(0)), f32(1))
            frac = min(max(f32(f32(1.0) - comp), cfg.reward_floor), f32(1))
            g = max(0, lround(f32(f32(cfg.grow_per_epoch) * frac)))
        return g

    def grow_local(self, p, fire_of, cfg):
        pre_l = self.layer[p] - 1
        if pre_l < 0:
            return -1
        b0, bn = self.layer_begin[pre_l], self.layer_count[pre_l]
        w = cfg.locality_window
        klo = min(max(int(math.ceil(f32(f32(self.pos[p] - w) * f32(bn - 1)))), 0), bn - 1)
        khi = min(max(int(math.floor(f32(f32(self.pos[p] + w) * f32(bn - 1)))), 0), bn - 1)
        best, best_fire = -1, -1
        for kk in range(klo, khi + 1):
            q = b0 + kk
            if self.connected(q, p):
                continue
            if fire_of(q) > best_fire:
                best_fire, best = fire_of(q), q
        return best

    def structural_update(self, fires, cfg: StructConfig, reward=1.0):
        """connectome.cpp:121-219: returns (pruned, grown, synapses)."""
        K0 = self.grow_target(cfg, reward)
        cand = [(abs(float(e[2])), i, k) for i in range(self.n) for k, e in enumerate(self.adj[i])
                if e[3] >= cfg.protect_rounds]
        K = min(K0, len(cand))
        rm = set()
        if K > 0:
            cand.sort()
            rm = {(i, k) for _, i, k in cand[:K]}
        freed, pruned = [], 0
        for i in range(self.n):
            keep = []
            for k, e in enumerate(self.adj[i]):
                if (i, k) in rm:
                    pruned += 1
                    freed.append(e[0])
                else:
                    keep.append(e)
            self.adj[i] = keep
        fires = np.asarray(fires)

        def fire_of(i):
            return int(fires[i]) if i < fires.shape[0] else 0

        grown = 0
        for p in freed:
            if grown >= pruned:
                break
            q = self.grow_local(p, fire_of, cfg)
            if q >= 0:
                self.adj[q].append([p, cfg.delay, cfg.w_grow_init, 0])
                grown += 1
        lo = self.layer_begin[1] if len(self.layer_begin) > 1 else 0
        hi = max(0, self.n - 1)
        attempts = 0
        max_attempts = cfg.max_attempts_mult * max(1, pruned)
        while grown < pruned and attempts < max_attempts:
            attempts += 1
            p = -1
            for _ in range(4):
                q = self.rng.uniform_int(lo, hi)
                if self.layer[q] == 0:
                    continue
                if p < 0 or fire_of(q) < fire_of(p):
                    p = q
            if p < 0:
                continue
            q = self.grow_local(p, fire_of, cfg)
            if q >= 0:
                self.adj[q].append([p, cfg.delay, cfg.w_grow_init, 0])
                grown += 1
        for a in self.adj:
            for e in a:
                if e[3] < AGE_CAP:
                    e[3] += 1
        self.last_fallback_attempts = attempts
        return pruned, grown, self.num_synapses()


# ---------------------------------------------------------------------------
# The unchanged reference's Connectome, through ref_shim.cpp
# ---------------------------------------------------------------------------

class RefConnectome:
    def __init__(self, layers, synapse_budget, delay, w_init, seed):
        from .oracle import ref_lib
        L = ref_lib()
        L.ref_con_layered_local.restype = C.c_void_p
        L.ref_con_layered_local.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float,
                                            C.c_uint64]
        L.ref_con_destroy.argtypes = [C.c_void_p]
        L.ref_con_num_synapses.argtypes = [C.c_void_p]
        L.ref_con_read.argtypes = [C.c_void_p] * 5
        L.ref_con_set_weights.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.ref_con_update.argtypes = ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_float,
                                      C.c_float, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float,
                                      C.c_float, C.c_void_p])
        self.L = L
        self.layers = np.ascontiguousarray(layers, np.int32)
        self.n = int(self.layers.sum())
        self.h = L.ref_con_layered_local(self.layers.ctypes.data, len(self.layers), int(synapse_budget),
                                         int(delay), float(w_init), int(seed))

    def to_csr(self):
        S = self.L.ref_con_num_synapses(self.h)
        row_ptr = np.zeros(self.n + 1, np.int32)
        post = np.zeros(max(1, S), np.int32)
        delay = np.zeros(max(1, S), np.int32)
        w = np.zeros(max(1, S), np.float32)
        self.L.ref_con_read(self.h, row_ptr.ctypes.data, post.ctypes.data, delay.ctypes.data,
                            w.ctypes.data)
        return row_ptr, post[:S], delay[:S], w[:S]

    def set_edge_weights(self, w):
        w = np.ascontiguousarray(w, np.float32)
        self.L.ref_con_set_weights(self.h, w.ctypes.data, int(w.shape[0]))

    def structural_update(self, fires, cfg: StructConfig, reward=1.0):
        fires = np.ascontiguousarray(fires, np.int64)
        out = np.zeros(3, np.int32)
        self.L.ref_con_update(self.h, fires.ctypes.data, int(fires.shape[0]), cfg.grow_per_epoch,
                              cfg.delay, float(cfg.w_grow_init), float(cfg.locality_window),
                              cfg.protect_rounds, cfg.max_attempts_mult, int(cfg.reward_modulated),
                              float(cfg.reward_chance), float(cfg.reward_floor), float(reward),
                              out.ctypes.data)
        return int(out[0]), int(out[1]), int(out[2])

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_con_destroy(self.h)
            self.h = None
