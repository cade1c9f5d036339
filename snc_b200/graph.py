"""Host-side spiking graph: the reference's ``SNNGraph`` CSR as numpy arrays.

Mirrors ``struct SNNGraph`` (include/snc/snn_graph.hpp:43-77): a CSR over
OUTGOING synapses (``row_ptr[N+1]``, ``post_ids[S]``, ``weights[S]``,
``delays[S]``, ``branch_ids[S]``) plus per-neuron ``role`` (0 internal, 1
input, 2 output), ``sign`` (+1/-1, Dale's sign on the pre neuron) and
``channel``.  Edges keep their insertion order inside each row
(``finalize``, src/graph/snn_graph.cpp:154-181); the backend relies on that
order for bit-exact delivery.

Also reads and writes the graph wire format of ``snc_export``
(src/bench/snc_export.cpp:107-123, python/snc/graph.py:11-24): little-endian
int32 ``magic 'SNCG', N, S, n_in, n_out, pre[S], post[S], delays[S], role[N],
channel[N]``.  Weights are not part of that format; ``save_sncg`` may append
an optional trailing section ``'SNCW', S, weights[S] (float32), sign[N]
(int32)`` that older readers ignore because they stop after ``channel``.
"""
from __future__ import annotations

import dataclasses

import numpy as np

INTERNAL, INPUT, OUTPUT = 0, 1, 2
SNCG_MAGIC = 0x534E4347  # 'SNCG'
SNCW_MAGIC = 0x534E4357  # 'SNCW' optional weights section


@dataclasses.dataclass
class SNNGraph:
    num_neurons: int
    row_ptr: np.ndarray   # int32 [N+1]
    post_ids: np.ndarray  # int32 [S]
    weights: np.ndarray   # float32 [S]
    delays: np.ndarray    # int32 [S]
    role: np.ndarray      # uint8 [N]
    sign: np.ndarray      # int8 [N]
    channel: np.ndarray   # int32 [N]
    branch_ids: np.ndarray | None = None  # uint8 [S], informational

    def __post_init__(self):
        self.row_ptr = np.ascontiguousarray(self.row_ptr, dtype=np.int32)
        self.post_ids = np.ascontiguousarray(self.post_ids, dtype=np.int32)
        self.weights = np.ascontiguousarray(self.weights, dtype=np.float32)
        self.delays = np.ascontiguousarray(self.delays, dtype=np.int32)
        self.role = np.ascontiguousarray(self.role, dtype=np.uint8)
        self.sign = np.ascontiguousarray(self.sign, dtype=np.int8)
        self.channel = np.ascontiguousarray(self.channel, dtype=np.int32)
        if self.branch_ids is None:
            self.branch_ids = np.zeros(self.post_ids.shape[0], dtype=np.uint8)
        self.rebuild_io_index()

    # -- SNNGraph::num_synapses / rebuild_io_index (snn_graph.cpp:13-28) -----
    @property
    def num_synapses(self) -> int:
        return int(self.post_ids.shape[0])

    def rebuild_io_index(self) -> None:
        self.input_neurons = np.nonzero(self.role == INPUT)[0].astype(np.int32)
        self.output_neurons = np.nonzero(self.role == OUTPUT)[0].astype(np.int32)
        ci = self.channel[self.input_neurons]
        co = self.channel[self.output_neurons]
        self.num_input_channels = int(ci.max()) + 1 if ci.size else 0
        self.num_output_channels = int(co.max()) + 1 if co.size else 0

    # -- SNNGraph::validate (snn_graph.cpp:30-56) ---------------------------
    def validate(self) -> str:
        """Return "" when the graph is structurally valid, else the reason."""
        n, m = self.num_neurons, self.num_synapses
        if n < 0:
            return "negative num_neurons"
        if self.row_ptr.shape[0] != n + 1:
            return "row_ptr size != num_neurons + 1"
        if not (self.role.shape[0] == n and self.sign.shape[0] == n and self.channel.shape[0] == n):
            return "per-neuron metadata size mismatch"
        if self.weights.shape[0] != m or self.delays.shape[0] != m or self.branch_ids.shape[0] != m:
            return "CSR column array size mismatch"
        if n > 0 and self.row_ptr[0] != 0:
            return "row_ptr[0] != 0"
        if self.row_ptr.shape[0] and self.row_ptr[-1] != m:
            return "row_ptr.back() != num_synapses"
        if n > 0 and np.any(np.diff(self.row_ptr) < 0):
            return "row_ptr not monotone"
        if m and (self.post_ids.min() < 0 or self.post_ids.max() >= n):
            return "post id out of range"
        if m and self.delays.min() < 1:
            return "delay < 1"
        return ""

    @property
    def max_delay(self) -> int:
        return max(1, int(self.delays.max())) if self.num_synapses else 1

    @property
    def ring_len(self) -> int:
        """Delay-ring length, one past the largest delay (cpu_backend.cpp:77-80)."""
        return self.max_delay + 1

    def pre_ids(self) -> np.ndarray:
        """CSR row owner of every synapse (snc_export.cpp:109-113)."""
        return np.repeat(np.arange(self.num_neurons, dtype=np.int32),
                         np.diff(self.row_ptr)).astype(np.int32)

    def stats(self) -> dict:
        """compute_stats (snn_graph.cpp:58-94) as a dict."""
        fo = np.diff(self.row_ptr)
        fi = np.bincount(self.post_ids, minlength=self.num_neurons) if self.num_synapses else np.zeros(self.num_neurons)
        n, m = self.num_neurons, self.num_synapses
        return {
            "num_neurons": n, "num_synapses": m,
            "num_inputs": int((self.role == INPUT).sum()),
            "num_outputs": int((self.role == OUTPUT).sum()),
            "avg_fan_out": m / n if n else 0.0, "max_fan_out": int(fo.max()) if n else 0,
            "avg_fan_in": m / n if n else 0.0, "max_fan_in": int(fi.max()) if n else 0,
            "fan_in_cv": float(fi.std() / fi.mean()) if m else 0.0,
            "avg_delay": float(self.delays.mean()) if m else 0.0,
            "density": m / (n * (n - 1)) if n > 1 else 0.0,
        }


def from_edges(num_neurons, pre, post, weights, delays, role, sign=None, channel=None) -> SNNGraph:
    """Build a CSR graph from an edge list, keeping the given edge order
    within each pre row (a stable sort by pre)."""
    pre = np.asarray(pre, dtype=np.int64)
    order = np.argsort(pre, kind="stable")
    counts = np.bincount(pre, minlength=num_neurons)
    row_ptr = np.zeros(num_neurons + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    if sign is None:
        sign = np.ones(num_neurons, dtype=np.int8)
    if channel is None:
        channel = np.full(num_neurons, -1, dtype=np.int32)
    return SNNGraph(num_neurons, row_ptr.astype(np.int32), np.asarray(post)[order],
                    np.asarray(weights, dtype=np.float32)[order], np.asarray(delays)[order],
                    role, sign, channel)


def load_graph(path):
    """python/snc/graph.py:11-24: read an SNCG file into the reference's dict
    (``N, S, n_in, n_out, pre, post, delays, role, channel``).  When the
    optional weights section is present, ``weights`` and ``sign`` are added."""
    with open(path, "rb") as f:
        magic, N, S, n_in, n_out = np.fromfile(f, dtype="<i4", count=5)
        if magic != SNCG_MAGIC:
            raise ValueError(f"{path}: bad magic 0x{int(magic) & 0xffffffff:08x}")
        pre = np.fromfile(f, dtype="<i4", count=S)
        post = np.fromfile(f, dtype="<i4", count=S)
        delays = np.fromfile(f, dtype="<i4", count=S)
        role = np.fromfile(f, dtype="<i4", count=N)
        channel = np.fromfile(f, dtype="<i4", count=N)
        d = {"N": int(N), "S": int(S), "n_in": int(n_in), "n_out": int(n_out),
             "pre": pre, "post": post, "delays": delays, "role": role, "channel": channel}
        tail = np.fromfile(f, dtype="<i4", count=2)
        if tail.shape[0] == 2 and tail[0] == SNCW_MAGIC and tail[1] == S:
            d["weights"] = np.fromfile(f, dtype="<f4", count=S)
            d["sign"] = np.fromfile(f, dtype="<i4", count=N)
    if pre.shape[0] != S or channel.shape[0] != N:
        raise ValueError(f"{path}: truncated SNCG file")
    return d


def graph_from_sncg(d) -> SNNGraph:
    """SNNGraph from a load_graph() dict (pre[] must be non-decreasing, as
    snc_export writes it).  Missing weights default to 1.0, sign to +1."""
    N, S = d["N"], d["S"]
    pre = np.asarray(d["pre"], dtype=np.int64)
    if S and np.any(np.diff(pre) < 0):
        raise ValueError("SNCG pre[] is not in CSR order")
    row_ptr = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(np.bincount(pre, minlength=N), out=row_ptr[1:])
    w = d.get("weights", np.ones(S, dtype=np.float32))
    sign = d.get("sign", np.ones(N, dtype=np.int32)).astype(np.int8)
    return SNNGraph(N, row_ptr.astype(np.int32), d["post"], w, d["delays"],
                    np.asarray(d["role"]).astype(np.uint8), sign, d["channel"])


def save_sncg(g: SNNGraph, path, with_weights=True) -> None:
    """Write the snc_export layout (snc_export.cpp:107-123); optionally append
    the weights section."""
    hdr = np.array([SNCG_MAGIC, g.num_neurons, g.num_synapses, g.num_input_channels,
                    g.num_output_channels], dtype="<i4")
    with open(path, "wb") as f:
        hdr.tofile(f)
        g.pre_ids().astype("<i4").tofile(f)
        g.post_ids.astype("<i4").tofile(f)
        g.delays.astype("<i4").tofile(f)
        g.role.astype("<i4").tofile(f)
        g.channel.astype("<i4").tofile(f)
        if with_weights:
            np.array([SNCW_MAGIC, g.num_synapses], dtype="<i4").tofile(f)
            g.weights.astype("<f4").tofile(f)
            g.sign.astype("<i4").tofile(f)


# InputEvent {int sample_id, channel_id, time; float amplitude}
# (include/snc/encoders.hpp:21-26), 16 bytes, same layout as the C ABI.
EVENT_DTYPE = np.dtype([("sample_id", "<i4"), ("channel_id", "<i4"),
                        ("time", "<i4"), ("amplitude", "<f4")])


def make_events(sample_id, channel_id, time, amplitude) -> np.ndarray:
    n = np.broadcast(sample_id, channel_id, time, amplitude).shape[0] if np.ndim(time) else 1
    ev = np.zeros(n, dtype=EVENT_DTYPE)
    ev["sample_id"], ev["channel_id"], ev["time"], ev["amplitude"] = sample_id, channel_id, time, amplitude
    return ev
