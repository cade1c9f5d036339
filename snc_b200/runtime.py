"""Runtime API: the reference's ``snc::forward`` / ``Backend`` surface over
the B200 kernels.

Mirrors include/snc/runtime.hpp:
  * ``Backend`` names (parse_backend / backend_name, cpu_backend.cpp:14-37):
    the reference's ``cuda-atomic`` / ``cuda-bucket`` / ``cuda-sort`` select
    this backend's ATOMIC / BUCKET / SORT delivery (a link-time drop-in, like
    the stub swap in CMakeLists.txt:60-65), and the new names
    ``b200-atomic`` / ``b200-bucket`` / ``b200-sort`` / ``b200-auto`` do the
    same explicitly.  ``cpu`` / ``openmp`` are the reference's own host
    backends and are not provided here.
  * ``LIFParams`` (runtime.hpp:34-39) plus ``reset_mode`` (1 = subtractive).
  * ``RunStats`` / ``ForwardResult`` (runtime.hpp:41-52).
  * ``forward(g, events, num_steps, lif, backend)`` (runtime.hpp:57-58): one
    sample through the autotuned path (persistent unless the tuner chose the
    plain per-step launches).  Unlike the reference, an unavailable device
    raises instead of silently falling back to the CPU.

Batched execution, device-resident inputs and results, and the autotuner are
additions: ``DeviceGraph``, ``DeviceInputs``, ``Run``, ``forward_batched``.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import sys

import numpy as np

from . import _lib
from ._lib import (MODE_ATOMIC, MODE_AUTO, MODE_BUCKET, MODE_SORT, PATH_AUTO, PATH_PERSISTENT,
                   PATH_PLAIN, RUN_FORCE_GRID, RUN_GRAPH, RUN_RASTER, RUN_VFINAL, check, lib,
                   ptr)
from .graph import EVENT_DTYPE, SNNGraph

BACKENDS = {
    "cuda-atomic": MODE_ATOMIC, "cuda-bucket": MODE_BUCKET, "cuda-sort": MODE_SORT,
    "b200-atomic": MODE_ATOMIC, "b200-bucket": MODE_BUCKET, "b200-sort": MODE_SORT,
    "b200-auto": MODE_AUTO,
}
MODE_NAMES = {MODE_ATOMIC: "atomic", MODE_BUCKET: "bucket", MODE_SORT: "sort", MODE_AUTO: "auto"}
PATH_NAMES = {PATH_PLAIN: "plain", PATH_PERSISTENT: "persistent", PATH_AUTO: "auto"}


def parse_backend(name: str) -> int:
    if name not in BACKENDS:
        raise ValueError(f"unknown backend {name!r} (choose from {sorted(BACKENDS)})")
    return BACKENDS[name]


def backend_name(mode: int) -> str:
    return "b200-" + MODE_NAMES[mode]


def backend_is_cuda(name: str) -> bool:
    return name in BACKENDS


def available() -> bool:
    """snc::cuda::available (cuda_backend.cu:181-184) for this backend."""
    return bool(lib().snc_b200_available())


def set_device(device: int) -> None:
    """Select the GPU for this thread's later calls into the library."""
    check(lib().snc_b200_set_device(int(device)), "set_device")


@dataclasses.dataclass
class LIFParams:
    threshold: float = 1.0
    decay: float = 0.9
    reset: float = 0.0
    refractory: int = 1
    reset_mode: int = 0  # 0: v = reset (reference), 1: v -= threshold

    def c(self):
        return _lib.Lif(self.threshold, self.decay, self.reset, self.refractory, self.reset_mode)


@dataclasses.dataclass
class RunStats:
    spikes: int = 0
    synaptic_events: int = 0
    overflow: int = 0
    ms: float = 0.0


@dataclasses.dataclass
class ForwardResult:
    logits: np.ndarray
    stats: RunStats
    used_backend: str


def graph_view(g: SNNGraph):
    """C view of a host graph (the arrays must outlive the call)."""
    return _lib.GraphView(g.num_neurons, g.num_synapses, ptr(g.row_ptr), ptr(g.post_ids),
                          ptr(g.weights), ptr(g.delays), ptr(g.role), ptr(g.sign), ptr(g.channel))


def _events(events) -> np.ndarray:
    if events is None:
        return np.zeros(0, dtype=EVENT_DTYPE)
    return np.ascontiguousarray(events, dtype=EVENT_DTYPE)


class DeviceGraph:
    """A graph uploaded once (snc_b200_graph_upload)."""

    def __init__(self, g: SNNGraph | None, _handle=None):
        self.host = g
        if _handle is None:
            view = graph_view(g)
            h = C.c_void_p()
            check(lib().snc_b200_graph_upload(C.byref(view), C.byref(h)), "graph_upload")
        else:
            h = _handle
        self.h = h
        self._info()

    @classmethod
    def from_sncg(cls, data) -> "DeviceGraph":
        """Upload an SNCG file (a path or its bytes) parsed and packed on the
        device (snc_b200_graph_upload_sncg)."""
        if not isinstance(data, (bytes, bytearray, memoryview)):
            with open(data, "rb") as f:
                data = f.read()
        buf = (C.c_char * len(data)).from_buffer_copy(data) if not isinstance(data, bytearray) \
            else (C.c_char * len(data)).from_buffer(data)
        h = C.c_void_p()
        check(lib().snc_b200_graph_upload_sncg(buf, len(data), C.byref(h)), "graph_upload_sncg")
        return cls(None, _handle=h)

    @classmethod
    def generate_grid(cls, spec: dict) -> "DeviceGraph":
        """Generate a grid graph on the device (snc_b200_graph_generate_grid)
        from a spec of snc_b200.workloads.grid_graph_spec."""
        p = _lib.GridGraph(spec["width"], spec["height"], spec["out_degree"], spec["long_range"],
                           spec["sigma"], spec["w_std"], spec["max_delay"], spec["max_draws"],
                           spec["seed"])
        acc = np.ascontiguousarray(spec["accept"], np.uint32)
        role = np.ascontiguousarray(spec["role"], np.uint8)
        sign = np.ascontiguousarray(spec["sign"], np.int8)
        ch = np.ascontiguousarray(spec["channel"], np.int32)
        h = C.c_void_p()
        check(lib().snc_b200_graph_generate_grid(C.byref(p), ptr(acc), ptr(role), ptr(sign), ptr(ch),
                                                 C.byref(h)), "graph_generate_grid")
        return cls(None, _handle=h)

    def blocks(self):
        """(block_size, num_blocks) of the graph's neuron-block partition."""
        bs, p = C.c_int32(), C.c_int32()
        check(lib().snc_b200_graph_layout(self.h, *([None] * 7), C.byref(bs), C.byref(p), None),
              "graph_layout")
        return bs.value, p.value

    def _info(self):
        n, s, r, no, ni = (C.c_int32() for _ in range(5))
        check(lib().snc_b200_graph_info(self.h, C.byref(n), C.byref(s), C.byref(r), C.byref(no),
                                        C.byref(ni)))
        self.N, self.S, self.ring_len, self.n_out, self.n_in = n.value, s.value, r.value, no.value, ni.value

    def release(self):
        if getattr(self, "h", None):
            lib().snc_b200_graph_release(self.h)
            self.h = None

    def __del__(self, _finalizing=sys.is_finalizing):
        # a default argument outlives the module globals cleared at exit
        if not _finalizing():  # the library may already be unloaded
            self.release()


class DeviceInputs:
    """An uploaded input schedule for a batch (snc_b200_inputs_upload)."""

    def __init__(self, dg: DeviceGraph, events, steps):
        ev = _events(events)
        self.steps = np.ascontiguousarray(steps, dtype=np.int32).reshape(-1)
        self.B = int(self.steps.shape[0])
        self.dg = dg
        h = C.c_void_p()
        check(lib().snc_b200_inputs_upload(dg.h, ptr(ev), ev.shape[0], self.B, ptr(self.steps),
                                           C.byref(h)), "inputs_upload")
        self.h = h
        self._info()

    def _info(self):
        nb, ne = C.c_int64(), C.c_int64()
        check(lib().snc_b200_inputs_info(self.h, C.byref(nb), C.byref(ne)), "inputs_info")
        self.device_bytes, self.entries = nb.value, ne.value

    ENCODERS = {"direct": _lib.ENCODER_DIRECT, "poisson": _lib.ENCODER_POISSON,
                "latency": _lib.ENCODER_LATENCY}

    @classmethod
    def encode(cls, dg: DeviceGraph, features, steps, encoder="poisson", gain=1.0, max_rate=0.5,
               threshold=0.0, seed=1) -> "DeviceInputs":
        """The schedule of a batch encoded on the device from its features
        [B, n_channels] (snc_b200_inputs_encode; encoders.cpp:25-71): direct
        and latency exactly as the reference encodes, poisson with
        Philox-4x32-10 draws."""
        f = np.ascontiguousarray(features, dtype=np.float32)
        if f.ndim != 2:
            raise ValueError("features must be [num_samples, n_channels]")
        self = cls.__new__(cls)
        self.steps = np.ascontiguousarray(steps, dtype=np.int32).reshape(-1)
        self.B = int(self.steps.shape[0])
        if f.shape[0] != self.B:
            raise ValueError("one row of features per sample")
        self.dg = dg
        enc = cls.ENCODERS[encoder] if isinstance(encoder, str) else int(encoder)
        h = C.c_void_p()
        check(lib().snc_b200_inputs_encode(dg.h, enc, ptr(f), f.shape[1], self.B, ptr(self.steps),
                                           gain, max_rate, threshold, int(seed), C.byref(h)),
              "inputs_encode")
        self.h = h
        self._info()
        return self

    def read(self):
        """The schedule back on the host: (sched_ptr [total steps + B],
        neuron [entries], drive [entries]) (snc_b200_inputs_read)."""
        ptr_ = np.zeros(int(self.steps.sum()) + self.B, np.int32)
        nid = np.zeros(max(1, self.entries), np.int32)
        ext = np.zeros(max(1, self.entries), np.float32)
        check(lib().snc_b200_inputs_read(self.h, ptr(ptr_), ptr(nid), ptr(ext)), "inputs_read")
        return ptr_, nid[:self.entries], ext[:self.entries]

    def release(self):
        if getattr(self, "h", None):
            lib().snc_b200_inputs_release(self.h)
            self.h = None

    def __del__(self, _finalizing=sys.is_finalizing):
        # a default argument outlives the module globals cleared at exit
        if not _finalizing():  # the library may already be unloaded
            self.release()


class Run:
    """Device-resident run of a batch; launch() is asynchronous on `stream`
    (a cudaStream_t as int, 0 = default stream), fetch() waits."""

    def __init__(self, dg: DeviceGraph, inputs: DeviceInputs, raster=False, vfinal=False,
                 cuda_graph=False, force_grid=False):
        self.dg, self.inputs = dg, inputs
        self.flags = ((RUN_RASTER if raster else 0) | (RUN_VFINAL if vfinal else 0) |
                      (RUN_GRAPH if cuda_graph else 0) | (RUN_FORCE_GRID if force_grid else 0))
        h = C.c_void_p()
        check(lib().snc_b200_run_create(dg.h, inputs.h, self.flags, C.byref(h)), "run_create")
        self.h = h

    def launch(self, lif: LIFParams, mode=MODE_SORT, path=PATH_PERSISTENT, stream=0):
        lf = lif.c()
        check(lib().snc_b200_run_launch(self.h, C.byref(lf), int(mode), int(path),
                                        C.c_void_p(stream) if stream else None), "run_launch")

    def set_readout(self, ro_decay):
        """Leaky readout units on the OUTPUT neurons (None or < 0: off)."""
        check(lib().snc_b200_run_set_readout(self.h, -1.0 if ro_decay is None else float(ro_decay)),
              "run_set_readout")

    def configure(self, tier=-1, block_threads=0, wave=0, ring_smem=-1, mode=MODE_SORT):
        """Fix the launch shape (snc_b200_run_configure); configure(None)
        semantics: call with no arguments to return to automatic shapes."""
        c = _lib.LaunchConfig(int(mode), PATH_PERSISTENT, int(tier), int(block_threads), int(wave),
                              int(ring_smem), 0.0)
        auto = tier == -1 and block_threads == 0 and wave == 0 and ring_smem == -1
        check(lib().snc_b200_run_configure(self.h, None if auto else C.byref(c)), "run_configure")

    def used(self):
        m, p = C.c_int(), C.c_int()
        check(lib().snc_b200_run_used(self.h, C.byref(m), C.byref(p)))
        return m.value, p.value

    def used_graph(self) -> bool:
        return lib().snc_b200_run_used_graph(self.h) == 1

    def fetch(self, raster=False, vfinal=False) -> dict:
        B, noc, N = self.inputs.B, self.dg.n_out, self.dg.N
        logits = np.zeros((B, max(noc, 1)), np.float32)
        spikes = np.zeros(B, np.int64)
        events = np.zeros(B, np.int64)
        W = (N + 31) // 32
        rast = np.zeros((int(self.inputs.steps.sum()), W), np.uint32) if raster else None
        v = np.zeros((B, N), np.float32) if vfinal else None
        st = _lib.RunStats()
        check(lib().snc_b200_run_fetch(self.h, ptr(logits), ptr(spikes), ptr(events), ptr(rast),
                                       ptr(v), C.byref(st)), "run_fetch")
        return {"logits": logits[:, :noc], "spikes": spikes, "events": events, "raster": rast,
                "v": v, "ms": st.ms, "total_spikes": st.spikes, "total_events": st.synaptic_events}

    def release(self):
        if getattr(self, "h", None):
            lib().snc_b200_run_release(self.h)
            self.h = None

    def __del__(self, _finalizing=sys.is_finalizing):
        # a default argument outlives the module globals cleared at exit
        if not _finalizing():  # the library may already be unloaded
            self.release()


def forward(g: SNNGraph, events, num_steps: int, lif: LIFParams, backend: str = "b200-sort",
            device_graph: DeviceGraph | None = None) -> ForwardResult:
    """snc::forward (runtime.hpp:57-58) for one sample on this backend."""
    mode = parse_backend(backend)
    ev = _events(events)
    lf = lif.c()
    noc = g.num_output_channels
    logits = np.zeros(max(noc, 1), np.float32)
    st = _lib.RunStats()
    view = graph_view(g)
    check(lib().snc_b200_forward(device_graph.h if device_graph else None,
                                 None if device_graph else C.byref(view), ptr(ev), ev.shape[0],
                                 int(num_steps), C.byref(lf), mode, ptr(logits), C.byref(st)),
          "forward")
    return ForwardResult(logits[:noc], RunStats(st.spikes, st.synaptic_events, st.overflow, st.ms),
                         backend_name(mode))


def forward_batched(dg: DeviceGraph, events, steps, lif: LIFParams, mode=MODE_SORT) -> dict:
    """Many samples (events carry sample_id) with uneven step counts in one
    persistent launch."""
    ev = _events(events)
    steps = np.ascontiguousarray(steps, dtype=np.int32)
    B = steps.shape[0]
    logits = np.zeros((B, max(dg.n_out, 1)), np.float32)
    spikes = np.zeros(B, np.int64)
    evs = np.zeros(B, np.int64)
    lf = lif.c()
    st = _lib.RunStats()
    check(lib().snc_b200_forward_batched(dg.h, ptr(ev), ev.shape[0], B, ptr(steps), C.byref(lf),
                                         int(mode), ptr(logits), ptr(spikes), ptr(evs),
                                         C.byref(st)), "forward_batched")
    return {"logits": logits[:, :dg.n_out], "spikes": spikes, "events": evs, "ms": st.ms}


def _shape_dict(c) -> dict:
    return {"mode": c.mode, "path": c.path, "tier": c.tier, "block_threads": c.block_threads,
            "wave": c.wave, "ring_smem": c.ring_smem, "ms": c.ms}


def autotune(dg: DeviceGraph, inputs: DeviceInputs, lif: LIFParams) -> dict:
    """Time every launch candidate (delivery mode x path x launch shape) on
    this graph and inputs; the winner is cached under the graph's content hash
    and the batch's shape and used by later MODE_AUTO / PATH_AUTO launches.
    Returns the winner (mode, path, tier, block_threads, wave, ring_smem, ms)
    with the list of timed candidates under "candidates"."""
    cands = (_lib.LaunchConfig * 64)()
    n, best = C.c_int32(), C.c_int32()
    lf = lif.c()
    check(lib().snc_b200_autotune_ex(dg.h, inputs.h, C.byref(lf), cands, 64, C.byref(n),
                                     C.byref(best)), "autotune")
    out = _shape_dict(cands[best.value])
    out["candidates"] = [_shape_dict(cands[i]) for i in range(min(64, n.value))]
    return out


def autotune_lookup(dg: DeviceGraph, inputs: DeviceInputs) -> dict | None:
    """The cached autotuner choice for this graph and batch shape, or None."""
    c = _lib.LaunchConfig()
    return _shape_dict(c) if lib().snc_b200_autotune_lookup(dg.h, inputs.h, C.byref(c)) == 1 else None


def probe_red_rate(n_slots: int, n_ops: int = 1 << 28) -> float:
    """Reductions per second this GPU completes at scattered addresses of a
    buffer of n_slots floats (snc_b200_probe_red_rate): the denominator of
    the ATOMIC delivery mode's roofline."""
    out = C.c_double()
    check(lib().snc_b200_probe_red_rate(int(n_slots), int(n_ops), C.byref(out)), "probe_red_rate")
    return float(out.value)
