#!/usr/bin/env python
"""Benchmark of the spiking substrate's forward hot path on B200.

Workload (one "step" = one full forward of it): rec100k, the large recurrent
substrate -- 100k LIF neurons on a 2-D torus, 10M synapses (95 local targets
with lognormal in-degree skew + 5 long-range per neuron), delays 1-30, 10% of
neurons Poisson-driven at 0.02 spikes/step, 1000 timesteps, batch 1.  Seeded
synthetic graph and inputs (snc_b200/workloads.py).

Our arm (default): the batched persistent path (one launch for all 1000
timesteps, CUDA-graph captured) in the delivery mode the autotuner picks.
  value  synaptic events/s, inputs and graph resident in HBM, L2 flushed
         (256 MiB write) before every timed step, CUDA-event device time.
  e2e    the same metric through snc_b200_forward_batched with host event
         arrays (in pinned host memory): host->device copy of the events,
         schedule build on the device, run and result read-back inside the
         timed region (wall clock).
Extra keys report sample-steps/s, the plain per-sample path, the
bit-identical SORT mode and the ratio persistent / plain; `configs` the
C1 (ff784) and C3 (audio700, uneven lengths) forwards on both paths and one
C3 e-prop minibatch beside its CPU restatement; `bptt` the BPTT step of the
custom kernels against the PyTorch-autograd bridge.

Reference arm (--impl reference): the reference's own CPU backend (compiled
from its sources into oracle/_ref, snc::forward with the OpenMP backend, all
host threads) on the same workload; rank 0 only.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
    python bench.py --leg bptt|bptt-custom|configs   # one extra leg alone (profiling)
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = ("synaptic events/s and sample-steps/s, batched vs plain path, 1 B200; BPTT step ms")
UNIT = "synaptic events/s"
WORKLOAD = "rec100k: 100k LIF, 10M synapses, delays 1-30, 1000 steps, batch 1"
HBM_FALLBACK_GBS = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=40)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--mode", default="auto", choices=["auto", "atomic", "bucket", "sort"])
    p.add_argument("--no-extra", action="store_true", help="skip the plain / sort / cpu legs")
    p.add_argument("--leg", choices=["bptt", "bptt-custom", "configs", "reference-gpu", "c3", "eprop"],
                   help="run only this extra leg on one GPU and print its JSON (for profiling)")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return HBM_FALLBACK_GBS, "fallback"


def alg_bytes(events, spikes, neuron_steps):
    """Algorithmic bytes of one forward: 12 B per synaptic event (post id,
    weight, delay), 8 B per spike (row bounds), 32 B per neuron-step
    (v, refr, drive, ring slot: read + write)."""
    return 12 * events + 8 * spikes + 32 * neuron_steps


class Clocks:
    """nvidia-smi clock / throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50", "-i", str(self.gpu_id)],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx = float(f[2])
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
            os.unlink(self.path)
        except Exception:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def reference_arm(args):
    rank, world, _ = dist_setup()
    if rank != 0:
        return 0
    from oracle import oracle as O
    from snc_b200 import workloads as W
    g = W.rec100k_graph(seed=1)
    ev, steps = W.rec100k_inputs(g, 1, 1000, seed=1)
    lif = W.lif_tau20()
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    if O.ref_available():
        kind = "reference"
        rg = O.RefGraph(g)
        fwd = lambda: rg.forward(ev, 1000, lif, backend="openmp")  # noqa: E731
    else:
        kind, threads = "port", 1
        fwd = lambda: O.forward(g, ev, 1000, lif)  # noqa: E731
    for _ in range(args.warmup):
        fwd()
    t_tot, e_tot = 0.0, 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r = fwd()
        t_tot += time.perf_counter() - t0
        e_tot += r["events"]
    value = e_tot / t_tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": {"workload": WORKLOAD, "backend": "openmp" if kind == "reference" else "serial"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": "full rec100k forward (1000 steps, batch 1) per step"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline(g, ev, lif, budget_s=10.0):
    """The reference CPU backend (serial), timed on this host on whole
    rec100k samples until ~budget_s of work."""
    from oracle import oracle as O
    if O.ref_available():
        kind = "reference"
        rg = O.RefGraph(g)
        fwd = lambda: rg.forward(ev, 1000, lif, backend="cpu")  # noqa: E731
    else:
        kind = "port"
        fwd = lambda: O.forward(g, ev, 1000, lif)  # noqa: E731
    n, t, e = 0, 0.0, 0
    while t < budget_s or n < 2:
        t0 = time.perf_counter()
        r = fwd()
        t += time.perf_counter() - t0
        e += r["events"]
        n += 1
    return {"value": e / t, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"{n} full rec100k forwards (1000 steps, batch 1), serial cpu backend; "
                      "the reference resets to 0 after a spike (it has no subtractive reset)"}, r


def parity_leg(dg, di, g, ev, lif, timed_mode, timed_out, ref_counts):
    """Results of the timed input checked against the CPU: the SORT mode's
    rasters, final potentials, logits and counts against the restatement
    (oracle, the benchmark's subtractive reset), the timed mode's spike and
    event totals against the same, and -- in the reference's own semantics
    (reset to 0, which its CPU backend implements; the timed cpu_baseline run
    of the same input) -- this backend's SORT counts and logits against the
    reference's serial backend."""
    from oracle import oracle as O
    from snc_b200 import runtime as R
    run = R.Run(dg, di, raster=True, vfinal=True, cuda_graph=True)
    run.launch(lif, mode=R.MODE_SORT, path=R.PATH_PERSISTENT)
    o = run.fetch(raster=True, vfinal=True)
    ref = O.forward_batched(g, ev, np.array([1000], np.int32), lif)
    exact = all(np.array_equal(o[k], ref[k]) for k in ("spikes", "events", "logits", "raster")) and \
        np.array_equal(o["v"].view(np.uint32), ref["v"].view(np.uint32))
    name = R.MODE_NAMES[timed_mode]
    rs, re_ = float(ref["spikes"][0]), float(ref["events"][0])
    ts, te = float(timed_out["total_spikes"]), float(timed_out["total_events"])
    out = {"input": "the timed rec100k input (seed 1)", "sort_exact_vs_oracle": bool(exact),
           f"{name}_spike_agreement_vs_oracle": min(ts, rs) / max(ts, rs, 1.0),
           f"{name}_event_agreement_vs_oracle": min(te, re_) / max(te, re_, 1.0)}
    if ref_counts is not None:
        lif0 = R.LIFParams(threshold=lif.threshold, decay=lif.decay, reset=lif.reset,
                           refractory=lif.refractory, reset_mode=0)
        run.launch(lif0, mode=R.MODE_SORT, path=R.PATH_PERSISTENT)
        o0 = run.fetch()
        out["sort_counts_equal_reference_serial"] = bool(
            int(o0["spikes"][0]) == ref_counts["spikes"] and int(o0["events"][0]) == ref_counts["events"]
            and np.array_equal(o0["logits"][0], ref_counts["logits"]))
        out["reference_semantics"] = "reset to 0 (the reference has no subtractive reset)"
    run.release()
    return out

def _time_cuda(fn, steps, warmup):
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        fn()
    t1.record()
    torch.cuda.synchronize()
    return t0.elapsed_time(t1) / steps


def c3_leg(mode="sort", launches=3):
    """C3 alone (audio700: 256 uneven samples, leaky readouts, persistent
    path under a CUDA graph) in one delivery mode, `launches` launches: the
    workload of the sample-per-CTA kernel's profiles."""
    from snc_b200 import runtime as R
    from snc_b200 import workloads as W
    g = W.audio700_graph()
    ev, steps = W.audio700_inputs(256)
    dg = R.DeviceGraph(g)
    di = R.DeviceInputs(dg, ev, steps)
    run = R.Run(dg, di, cuda_graph=True)
    run.set_readout(0.9)
    m = {"atomic": R.MODE_ATOMIC, "sort": R.MODE_SORT}[mode]
    ms = []
    for _ in range(launches):
        run.launch(W.lif_tau20(), mode=m, path=R.PATH_PERSISTENT)
        ms.append(run.fetch()["ms"])
    return {"mode": mode, "ms": ms}


def config_legs(reps=3):
    """The other forward configurations and the e-prop update:
    C1 (ff784: 784-256-10, 64 samples x 50 steps) and C3 (audio700: 700 input
    channels, 1024 recurrent, 20 outputs, 256 samples of 50-1000 steps) on the
    persistent and the plain path in ATOMIC and SORT delivery (device time,
    best of `reps`; C3's 20 outputs are leaky readout units with decay 0.9,
    the persistent launches go through a CUDA graph), and one C3 e-prop minibatch (32 samples, the graph's
    weights, forward with eligibility + weight update, SORT) beside the CPU
    restatement of the same minibatch (one core) with the largest weight
    difference between them."""
    import numpy as np
    import torch
    from oracle import oracle as O
    from snc_b200 import eprop as EP
    from snc_b200 import runtime as R
    from snc_b200 import workloads as W
    lif = W.lif_tau20()
    out = {}
    for name, g, (ev, steps) in (("C1_ff784", W.ff784_graph(), W.ff784_inputs(64)),
                                 ("C3_audio700", W.audio700_graph(), W.audio700_inputs(256))):
        dg = R.DeviceGraph(g)
        di = R.DeviceInputs(dg, ev, steps)
        run = R.Run(dg, di, cuda_graph=True)  # the persistent launch goes through a CUDA graph
        if name.startswith("C3"):
            run.set_readout(0.9)  # C3's 20 leaky readout units
        ss = int(np.sum(steps))
        leg = {"samples": int(len(steps)), "sample_steps": ss}
        for m in (R.MODE_ATOMIC, R.MODE_SORT):
            for p in (R.PATH_PERSISTENT, R.PATH_PLAIN):
                ms = []
                for _ in range(reps + 1):
                    run.launch(lif, mode=m, path=p)
                    o = run.fetch()
                    ms.append(o["ms"])
                best = min(ms[1:])
                leg[f"{R.MODE_NAMES[m]}_{R.PATH_NAMES[p]}"] = {
                    "ms": best, "events_per_s": o["total_events"] / (best / 1e3),
                    "sample_steps_per_s": ss / (best / 1e3),
                    "cuda_graph": bool(run.used_graph())}
        leg["persistent_vs_plain_sort"] = leg["sort_plain"]["ms"] / leg["sort_persistent"]["ms"]
        out[name] = leg
        run.release()
        di.release()
        dg.release()
    # input encoding of the C3 batch (256 samples x 700 channels, Poisson):
    # on the device from the features vs the reference's encode() on the host
    # followed by the upload of its events (both build the device schedule)
    g = W.audio700_graph()
    _, steps = W.audio700_inputs(256)
    feats = np.minimum(np.random.default_rng(3).lognormal(np.log(0.01) - 0.5, 1.0, (256, 700)),
                       1.0).astype(np.float32)
    dg = R.DeviceGraph(g)
    dev = []
    for _ in range(reps + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        di = R.DeviceInputs.encode(dg, feats, steps, encoder="poisson", max_rate=1.0, seed=1)
        dev.append(1e3 * (time.perf_counter() - t0))
        n_dev = di.entries
        di.release()
    leg = {"samples": 256, "channels": 700, "sample_steps": int(np.sum(steps)),
           "device_ms": min(dev[1:]), "entries": int(n_dev)}
    if O.ref_available():
        t0 = time.perf_counter()
        ev = np.concatenate([O.ref_encode("poisson", feats[b], int(steps[b]), max_rate=1.0,
                                          seed=1 + b, sample_id=b) for b in range(256)])
        t1 = time.perf_counter()
        di = R.DeviceInputs(dg, ev, steps)
        t2 = time.perf_counter()
        leg.update({"host_encode_ms": 1e3 * (t1 - t0), "host_upload_ms": 1e3 * (t2 - t1),
                    "host_entries": int(di.entries)})
        di.release()
    out["encode_C3"] = leg
    dg.release()
    out["eprop_C3"] = eprop_leg(lif, reps)
    return out


def eprop_leg(lif=None, reps=3):
    """One C3 e-prop minibatch (32 samples, the graph's own weights) with
    SORT and ATOMIC delivery beside the CPU restatement (also `--leg eprop`,
    for profiling)."""
    import torch
    from oracle import oracle as O
    from snc_b200 import eprop as EP
    from snc_b200 import runtime as R
    from snc_b200 import workloads as W
    lif = lif or W.lif_tau20()
    g = W.audio700_graph()
    ev, steps = W.audio700_inputs(32)
    labels = np.random.default_rng(5).integers(0, g.num_output_channels, 32).astype(np.int32)
    cfg = EP.TrainConfig(lif=lif, lr=1.0, trace_decay=0.95, mode=R.MODE_SORT)
    # the graph's own (signed) weights: the C3 substrate's firing regime
    sess = EP.create(g, cfg, 32, weights=np.asarray(g.weights, np.float32) *
                     np.asarray(g.sign, np.float32)[g.pre_ids()])
    w0 = sess.get_weights()
    dev_ms, wall_ms = [], []
    for i in range(reps + 1):
        sess.set_weights(w0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        o = sess.run_batch(ev, steps, labels, train=True)
        wall_ms.append(1e3 * (time.perf_counter() - t0))
        dev_ms.append(o["ms"])
    w_gpu = sess.get_weights()
    # the same minibatch with unordered (atomic) delivery, as the reference's
    # GPU trainer delivers
    cfg_a = EP.TrainConfig(lif=lif, lr=1.0, trace_decay=0.95, mode=R.MODE_ATOMIC)
    sess_a = EP.create(g, cfg_a, 32, weights=w0)
    atomic_ms = []
    for i in range(reps + 1):
        sess_a.set_weights(w0)
        atomic_ms.append(sess_a.run_batch(ev, steps, labels, train=True)["ms"])
    sess_a.release()
    t0 = time.perf_counter()
    ref = O.eprop_batch(g, w0, ev, steps, lif, trace_decay=0.95, gamma=cfg.surrogate_scale,
                        lr=cfg.lr, w_max=cfg.w_max, train_hidden=cfg.train_hidden,
                        bmat=sess.feedback, labels=labels, train=True)
    cpu_ms = 1e3 * (time.perf_counter() - t0)
    diff = float(np.abs(w_gpu - ref["w"]).max() / max(1e-30, float(np.abs(ref["w"]).max())))
    ss = int(np.sum(steps))
    res = {"batch": 32, "sample_steps": ss, "device_ms": min(dev_ms[1:]),
           "wall_ms": min(wall_ms[1:]), "synaptic_events": int(o["events"]),
           "events_per_s": o["events"] / (min(dev_ms[1:]) / 1e3),
           "device_ms_atomic_delivery": min(atomic_ms[1:]),
           "samples_per_s": 32 / (min(wall_ms[1:]) / 1e3),
           "cpu_port_ms": cpu_ms, "cpu_cores": 1,
           "max_rel_weight_diff": diff}
    sess.release()
    return res


def graph_build_leg(g, host_build_s):
    """Getting the 10M-synapse graph onto the device, three ways: the host
    numpy build of rec100k (timed by the caller) followed by the upload of
    its arrays (validation, hashing, device packing); the same graph's SNCG
    file image parsed and packed on the device; and a graph of the same
    shape (100k neurons on a 400 x 250 torus, 100 synapses each, delays 1-30)
    generated on the device by the counter-based generator (its per-neuron
    spec built on the host first).  Wall times of the calls."""
    import torch
    from snc_b200 import graph as G
    from snc_b200 import runtime as R
    from snc_b200 import workloads as W
    out = {"host_numpy_build_s": host_build_s, "synapses": int(g.num_synapses)}
    for name, fn in (("upload_host_arrays_ms", lambda: R.DeviceGraph(g)),):
        t0 = time.perf_counter()
        dg = fn()
        torch.cuda.synchronize()
        out[name] = 1e3 * (time.perf_counter() - t0)
        dg.release()
    with tempfile.NamedTemporaryFile(suffix=".sncg") as f:
        G.save_sncg(g, f.name)
        data = open(f.name, "rb").read()
    ms = []
    for _ in range(2):
        t0 = time.perf_counter()
        dg = R.DeviceGraph.from_sncg(data)
        torch.cuda.synchronize()
        ms.append(1e3 * (time.perf_counter() - t0))
        dg.release()
    out["sncg_device_ingest_ms"] = min(ms)
    out["sncg_bytes"] = len(data)
    t0 = time.perf_counter()
    spec = W.grid_graph_spec(seed=1)
    out["grid_spec_host_ms"] = 1e3 * (time.perf_counter() - t0)
    ms = []
    for _ in range(2):
        t0 = time.perf_counter()
        dg = R.DeviceGraph.generate_grid(spec)
        torch.cuda.synchronize()
        ms.append(1e3 * (time.perf_counter() - t0))
        S = dg.S
        dg.release()
    out["device_generate_ms"] = min(ms)
    out["device_generate_synapses"] = int(S)
    return out


REF_GPU_LIB = os.path.join(ROOT, "snc_b200", "adapter", "_build", "libsncref_gpu.so")
REF_BACKENDS = {"atomic": 2, "bucket": 3, "sort": 4}  # the reference's Backend::Cuda* values


class RefGpu:
    """The reference's own GPU implementation -- src/runtime/cuda_backend.cu
    and src/training/cuda_trainer.cu unchanged, compiled for sm_100a with its
    CPU sources into snc_b200/adapter/_build/libsncref_gpu.so (make -C
    snc_b200/adapter side) -- reached through its public API (snc::forward
    with the cuda-* backends, snc::cudatrain) by ref_gpu_shim.cpp."""

    def __init__(self):
        import ctypes as C
        self.C = C
        self.L = C.CDLL(REF_GPU_LIB)
        P, I, F = C.c_void_p, C.c_int, C.c_float
        self.L.refgpu_graph_create.restype = P
        self.L.refgpu_graph_create.argtypes = [I, I] + [P] * 7
        self.L.refgpu_graph_destroy.argtypes = [P]
        self.L.refgpu_available.restype = I
        self.L.refgpu_forward.restype = C.c_double
        self.L.refgpu_forward.argtypes = [P, P, C.c_int64, I, F, F, F, I, I, P, P, P, P, P]
        self.L.refgpu_train.restype = C.c_double
        self.L.refgpu_train.argtypes = [P, I, F, F, F, I, F, F, F, I, I, I, P, P, I, I, P, P]

    def graph(self, g):
        p = lambda a: a.ctypes.data  # noqa: E731
        arrs = [np.ascontiguousarray(a, t) for a, t in
                ((g.row_ptr, np.int32), (g.post_ids, np.int32), (g.weights, np.float32),
                 (g.delays, np.int32), (g.role, np.uint8), (g.sign, np.int8), (g.channel, np.int32))]
        h = self.L.refgpu_graph_create(g.num_neurons, g.num_synapses, *[p(a) for a in arrs])
        return h, arrs

    def forward(self, h, n_out, ev, steps, lif, mode):
        C = self.C
        ev = np.ascontiguousarray(ev)
        logits = np.zeros(max(1, n_out), np.float32)
        sp, en, used, wall = C.c_int64(), C.c_int64(), C.c_int(), C.c_double()
        ms = self.L.refgpu_forward(h, ev.ctypes.data, ev.shape[0], int(steps), lif.threshold, lif.decay,
                                   lif.reset, lif.refractory, REF_BACKENDS[mode], logits.ctypes.data,
                                   C.byref(sp), C.byref(en), C.byref(used), C.byref(wall))
        if used.value != REF_BACKENDS[mode]:
            raise RuntimeError(f"reference cuda-{mode} fell back to the CPU")
        return {"ms": ms, "wall_ms": wall.value, "spikes": sp.value, "events": en.value}


def reference_gpu_leg(budget_s=40.0, g_c2=None):
    """The reference's GPU kernels beside this backend's on the same B200 and
    the same inputs, in the reference's LIF semantics (reset to 0: it has no
    subtractive reset), forward of every delivery mode:
      C1 ff784 (64 samples x 50 steps), C2 rec100k (1 x 1000 steps),
      C3 audio700 (the first 32 of the 256 uneven samples; the reference runs
      one sample per call) --
    the reference per sample through snc::forward (its RunStats.ms: the step
    loop, launches included; and the wall time of the call, which also
    uploads the graph and frees it), this backend's plain path (one sample
    per launch sequence, like the reference) and persistent path (device
    time).  Then one e-prop minibatch on C3's graph: the reference's
    cudatrain::train_epoch on 32 samples of mean length (its trainer needs
    one length per session) beside this backend's minibatch on the same
    samples' uneven lengths, as sample-steps per second."""
    if not os.path.exists(REF_GPU_LIB):
        return {"unavailable": "snc_b200/adapter/_build/libsncref_gpu.so not built "
                               "(make -C snc_b200/adapter side needs the reference sources)"}
    import torch
    from snc_b200 import eprop as EP
    from snc_b200 import runtime as R
    from snc_b200 import workloads as W
    ref = RefGpu()
    if ref.L.refgpu_available() != 1:
        return {"unavailable": "the reference's cuda::available() is false"}
    lif0 = W.lif_tau20()
    lif = R.LIFParams(threshold=lif0.threshold, decay=lif0.decay, reset=0.0,
                      refractory=lif0.refractory, reset_mode=0)
    out = {"lif": "threshold 1, decay exp(-1/20), reset to 0, refractory 0 (the reference's semantics)"}
    t_start = time.perf_counter()
    for name, make_g, make_in in (
            ("C1_ff784", W.ff784_graph, lambda g: W.ff784_inputs(64)),
            ("C2_rec100k", lambda: g_c2 if g_c2 is not None else W.rec100k_graph(seed=1),
             lambda g: W.rec100k_inputs(g, 1, 1000, seed=1)),
            ("C3_audio700_32", W.audio700_graph, lambda g: W.audio700_inputs(256))):
        g = make_g()
        ev, steps = make_in(g)
        if name.startswith("C3"):
            keep = np.arange(32)
            ev = ev[np.isin(ev["sample_id"], keep)]
            steps = steps[:32]
        B = len(steps)
        per = [ev[ev["sample_id"] == b] for b in range(B)]
        h, _keep = ref.graph(g)
        dg = R.DeviceGraph(g)
        di = R.DeviceInputs(dg, ev, steps)
        run = R.Run(dg, di, cuda_graph=True)
        leg = {"samples": B, "sample_steps": int(np.sum(steps))}
        for mode in ("atomic", "bucket", "sort"):
            if time.perf_counter() - t_start > budget_s:
                leg[f"reference_{mode}"] = {"skipped": f"leg budget {budget_s:.0f} s spent"}
                continue
            loop_ms = wall_ms = 0.0
            sp = en = 0
            for b in range(B):
                r = ref.forward(h, g.num_output_channels, per[b], steps[b], lif, mode)
                loop_ms += r["ms"]
                wall_ms += r["wall_ms"]
                sp += r["spikes"]
                en += r["events"]
            leg[f"reference_{mode}"] = {"loop_ms": loop_ms, "call_ms": wall_ms, "spikes": sp,
                                        "events": en, "events_per_s_loop": en / (loop_ms / 1e3)}
            m = {"atomic": R.MODE_ATOMIC, "bucket": R.MODE_BUCKET, "sort": R.MODE_SORT}[mode]
            for p in (R.PATH_PLAIN, R.PATH_PERSISTENT):
                ms = []
                for _ in range(3):
                    run.launch(lif, mode=m, path=p)
                    o = run.fetch()
                    ms.append(o["ms"])
                best = min(ms[1:])
                leg[f"b200_{mode}_{R.PATH_NAMES[p]}"] = {
                    "ms": best, "spikes": int(o["total_spikes"]), "events": int(o["total_events"]),
                    "events_per_s": o["total_events"] / (best / 1e3),
                    "speedup_vs_reference_loop": loop_ms / best}
        out[name] = leg
        run.release()
        di.release()
        dg.release()
        ref.L.refgpu_graph_destroy(h)
    # e-prop minibatch on C3's graph
    g = W.audio700_graph()
    ev, steps = W.audio700_inputs(32)
    T_mean = int(round(float(np.mean(steps))))
    feats = np.minimum(np.random.default_rng(3).lognormal(np.log(0.01) - 0.5, 1.0, (32, 700)),
                       1.0).astype(np.float32)
    labels = np.random.default_rng(5).integers(0, g.num_output_channels, 32).astype(np.int32)
    h, _keep = ref.graph(g)
    C = ref.C
    sp, en = C.c_int64(), C.c_int64()
    ref.L.refgpu_train(h, T_mean, lif.threshold, lif.decay, lif.reset, lif.refractory, 1.0, 1.0, 0.3,
                       32, 700, g.num_output_channels, feats.ctypes.data, labels.ctypes.data, 32, 1,
                       C.byref(sp), C.byref(en))  # warm-up epoch
    ms_ref = ref.L.refgpu_train(h, T_mean, lif.threshold, lif.decay, lif.reset, lif.refractory, 1.0,
                                1.0, 0.3, 32, 700, g.num_output_channels, feats.ctypes.data,
                                labels.ctypes.data, 32, 3, C.byref(sp), C.byref(en)) / 3
    ref.L.refgpu_graph_destroy(h)
    cfg = EP.TrainConfig(lif=lif, lr=1.0, trace_decay=lif.decay, mode=R.MODE_ATOMIC)
    sess = EP.create(g, cfg, 32)
    wall = []
    for _ in range(4):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sess.run_batch(ev, steps, labels, train=True)
        wall.append(1e3 * (time.perf_counter() - t0))
    sess.release()
    ss_ref, ss_ours = 32 * T_mean, int(np.sum(steps))
    out["eprop_C3_minibatch32"] = {
        "reference_epoch_ms": ms_ref, "reference_T": T_mean,
        "reference_sample_steps_per_s": ss_ref / (ms_ref / 1e3),
        "b200_wall_ms": min(wall[1:]), "b200_sample_steps": ss_ours,
        "b200_sample_steps_per_s": ss_ours / (min(wall[1:]) / 1e3),
        "note": "reference: Poisson drawn on the GPU by cuRAND, one T per session; "
                "b200: host-encoded events, uneven T, atomic delivery"}
    return out


def bptt_leg(steps=3, warmup=2, lm=True, with_reference=True):
    """BPTT step (forward + backward) of the custom kernels against the
    PyTorch-autograd bridge (oracle/bptt_ref.py, the reference bridge's model
    with per-synapse delays) on the same GPU.
      mnist-like: 784 Poisson -> 512 -> 512 LIF (local sparse, delays 1-4)
                  -> 10 leaky readout, T=100, B=128, checkpoint every 10.
      char-LM:    4096 recurrent LIF, fan-in 64, delays 1-8, 96-symbol
                  Zipf tokens, B=64, T=256, checkpoint every 16.
    with_reference=False times the custom steps alone (no bridge, no
    gradient comparison)."""
    import torch
    import torch.nn.functional as F

    from oracle import bptt_ref as BR
    from snc_b200 import bptt as BP
    from snc_b200 import workloads as W
    out = {}
    c4 = W.bptt_mnist_like()
    dev = "cuda"
    model = BP.DelayedSNN(c4["N"], c4["pre"], c4["post"], c4["delays"], c4["n_in"],
                          c4["readout_ids"], 10, thr=1.0, decay=0.95, surrogate_scale=25.0,
                          ckpt_every=10).to(dev)
    x = torch.as_tensor(c4["spikes"], device=dev)
    y = torch.as_tensor(c4["labels"], device=dev)

    def custom():
        model.zero_grad(set_to_none=True)
        F.cross_entropy(model(x), y).backward()

    order = np.argsort(c4["pre"], kind="stable")
    w_ref = model.w.detach().clone().requires_grad_(True)
    wro = model.readout.weight.detach().clone().requires_grad_(True)
    bro = model.readout.bias.detach().clone().requires_grad_(True)
    pre = torch.as_tensor(c4["pre"], device=dev).long()
    post = torch.as_tensor(c4["post"], device=dev).long()
    dl = torch.as_tensor(c4["delays"], device=dev).long()
    rid = torch.as_tensor(c4["readout_ids"], device=dev).long()

    def reference():
        for p in (w_ref, wro, bro):
            p.grad = None
        ext = torch.zeros(x.shape[0], x.shape[1], c4["N"], device=dev)
        ext[:, :, :c4["n_in"]] = x
        s = BR.core_forward(w_ref, ext, pre, post, dl, 1.0, 0.95, 25.0)
        F.cross_entropy(BR.leaky_readout(s, wro, bro, rid, 0.9), y).backward()

    del order
    ms_c = _time_cuda(custom, steps, warmup)
    out["mnist_like"] = {"custom_ms": ms_c, "T": 100, "B": 128, "synapses": int(len(c4["pre"]))}
    if with_reference:
        ms_r = _time_cuda(reference, steps, warmup)
        rel = float((model.w.grad - w_ref.grad).abs().max() / w_ref.grad.abs().max().clamp_min(1e-30))
        out["mnist_like"].update({"autograd_ms": ms_r, "speedup": ms_r / ms_c, "grad_rel_err": rel})
    if lm:
        c5 = W.char_lm()
        torch.manual_seed(0)
        net = BP.SpikingLM(c5["vocab"], c5["H"], c5["pre"], c5["post"], c5["delays"], w_scale=2.0,
                           ckpt_every=16).to(dev)
        xt = torch.as_tensor(c5["x"], device=dev)
        yt = torch.as_tensor(c5["y"], device=dev)

        def lm_custom():
            net.zero_grad(set_to_none=True)
            F.cross_entropy(net(xt).reshape(-1, c5["vocab"]), yt.reshape(-1)).backward()

        pre5 = torch.as_tensor(c5["pre"], device=dev).long()
        post5 = torch.as_tensor(c5["post"], device=dev).long()
        d5 = torch.as_tensor(c5["delays"], device=dev).long()
        emb = net.embed.weight.detach().clone().requires_grad_(True)
        wr = net.w_rec.detach().clone().requires_grad_(True)
        wo = net.readout.weight.detach().clone().requires_grad_(True)
        bo = net.readout.bias.detach().clone().requires_grad_(True)

        def lm_reference():
            for p in (emb, wr, wo, bo):
                p.grad = None
            s = BR.core_forward(wr, emb[xt].transpose(0, 1), pre5, post5, d5, 1.0, 0.95, 25.0)
            r = torch.zeros(xt.shape[0], c5["H"], device=dev)
            rs = []
            for t in range(s.shape[0]):
                r = 0.9 * r + s[t]
                rs.append(r)
            lg = F.linear(torch.stack(rs, 1), wo, bo)
            F.cross_entropy(lg.reshape(-1, c5["vocab"]), yt.reshape(-1)).backward()

        ms_c5 = _time_cuda(lm_custom, 2, 1)
        out["char_lm"] = {"custom_ms": ms_c5, "T": 256, "B": 64, "synapses": int(len(c5["pre"])),
                          "tokens_per_s": 64 * 256 / (ms_c5 / 1e3)}
        if with_reference:
            ms_r5 = _time_cuda(lm_reference, 1, 1)
            rel5 = float((net.w_rec.grad - wr.grad).abs().max() / wr.grad.abs().max().clamp_min(1e-30))
            out["char_lm"].update({"autograd_ms": ms_r5, "speedup": ms_r5 / ms_c5, "grad_rel_err": rel5})
    return out


def our_arm(args):
    import torch
    rank, world, local = dist_setup()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    from snc_b200 import runtime as R
    from snc_b200 import workloads as W
    R.set_device(local)
    lif = W.lif_tau20()
    t_build = time.perf_counter()
    g = W.rec100k_graph(seed=1)
    t_build = time.perf_counter() - t_build
    ev, steps = W.rec100k_inputs(g, 1, 1000, seed=1 + rank)
    dg = R.DeviceGraph(g)
    di = R.DeviceInputs(dg, ev, steps)
    modes = {"atomic": R.MODE_ATOMIC, "bucket": R.MODE_BUCKET, "sort": R.MODE_SORT}
    if args.mode == "auto":
        tuned = R.autotune(dg, di, lif)
        mode = tuned["mode"] if tuned["path"] == R.PATH_PERSISTENT else R.MODE_BUCKET
    else:
        mode = modes[args.mode]
    run = R.Run(dg, di, cuda_graph=True)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    last = {}

    def timed(run_, mode_, path_, k):
        ms, ev_n, sp_n = [], 0, 0
        for _ in range(k):
            flush.zero_()
            run_.launch(lif, mode=mode_, path=path_)
            o = run_.fetch()
            ms.append(o["ms"])
            ev_n += o["total_events"]
            sp_n += o["total_spikes"]
            last["o"] = o
        return ms, ev_n, sp_n

    timed(run, mode, R.PATH_PERSISTENT, args.warmup)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    dev_props = torch.cuda.get_device_properties(local)
    clocks = Clocks(f"GPU-{dev_props.uuid}" if getattr(dev_props, "uuid", None) else local)
    clocks.start()
    ms, ev_n, sp_n = timed(run, mode, R.PATH_PERSISTENT, args.steps)
    torch.cuda.synchronize()
    clk = clocks.stop()
    timed_out = last["o"]
    used_graph = run.used_graph()
    tot_ms = float(sum(ms))
    if dist:
        t = torch.tensor([tot_ms, float(ev_n)], dtype=torch.float64, device="cuda")
        mx = t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        tot_ms_max, ev_all = float(mx[0]), float(t[1])
    else:
        tot_ms_max, ev_all = tot_ms, float(ev_n)
    value = ev_all / (tot_ms_max / 1e3)
    ms_per_step = tot_ms_max / args.steps

    # end to end through the C ABI with host buffers: the events sit in pinned
    # host memory, as a caller streaming inputs to the GPU keeps them
    pin = torch.empty(max(1, ev.nbytes), dtype=torch.uint8, pin_memory=True)
    ev_host = pin.numpy()[:ev.nbytes].view(ev.dtype)
    ev_host[:] = ev
    e2e_t, e2e_ev = 0.0, 0
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        o = R.forward_batched(dg, ev_host, steps, lif, mode=mode)
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            e2e_t += dt
            e2e_ev += int(o["events"].sum())
    if dist:
        t = torch.tensor([e2e_t, float(e2e_ev)], dtype=torch.float64, device="cuda")
        mx = t.clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        e2e_t, e2e_ev = float(mx[0]), float(t[1])
    e2e = {"value": e2e_ev / e2e_t, "unit": UNIT, "h2d_bytes_per_step": int(di.device_bytes),
           "d2h_bytes_per_step": int(4 * max(1, dg.n_out) + 16 + 4),
           "graph": "resident (uploaded once before the timed region; events, schedule build, "
                    "run and results inside it)",
           "host_events": "pinned"}

    extra = {}
    if not args.no_extra:
        k2 = max(2, min(5, args.steps))
        for name, m, p in (("plain_sort", R.MODE_SORT, R.PATH_PLAIN),
                           ("persistent_sort", R.MODE_SORT, R.PATH_PERSISTENT),
                           ("plain_best", mode, R.PATH_PLAIN)):
            r2 = R.Run(dg, di, cuda_graph=(p == R.PATH_PERSISTENT))
            timed(r2, m, p, 1)
            ms2, ev2, _ = timed(r2, m, p, k2)
            extra[name] = {"events_per_s": ev2 / (sum(ms2) / 1e3), "ms_per_step": sum(ms2) / k2,
                           "mode": R.MODE_NAMES[m]}
            r2.release()
        extra["persistent_vs_plain_sort"] = extra["persistent_sort"]["events_per_s"] / extra["plain_sort"]["events_per_s"]
        # the persistent loop's synchronisation floor: the same graph, launch
        # shape, mode and 1000 steps with no drive (nothing fires: integration
        # and the grid barrier of every step, no delivery)
        di0 = R.DeviceInputs(dg, np.zeros(0, dtype=W.EVENT_DTYPE), steps)
        r0 = R.Run(dg, di0, cuda_graph=True)
        timed(r0, mode, R.PATH_PERSISTENT, 2)
        ms0, _, sp0 = timed(r0, mode, R.PATH_PERSISTENT, k2)
        r0.release()
        di0.release()
        floor_us = 1e3 * sum(ms0) / k2 / 1000
        actual_us = 1e3 * ms_per_step / 1000
        extra["sync_floor"] = {"us_per_step": floor_us, "actual_us_per_step": actual_us,
                               "floor_over_actual": floor_us / actual_us, "spikes": int(sp0),
                               "mode": R.MODE_NAMES[mode]}

    peak, peak_kind = peaks()
    per_launch_bytes = alg_bytes(ev_n / args.steps, sp_n / args.steps, g.num_neurons * 1000)
    achieved = per_launch_bytes / (tot_ms / args.steps / 1e3) / 1e9
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "rec100k_traffic.json")
    if os.path.exists(tpath):
        try:
            with open(tpath) as f:
                traffic = json.load(f).get(R.MODE_NAMES[mode])
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                "kernel": "k_tier_g", "bytes_per_launch": per_launch_bytes,
                "bytes_per_launch_with_ring_rmw": per_launch_bytes + 8 * ev_n / args.steps}
    # the atomic half: the ATOMIC delivery mode (one red.global.add.f32 per
    # synaptic event into an L2-resident ring) against the measured rate of
    # scattered reductions into a buffer of the ring's size
    ra = R.Run(dg, di, cuda_graph=True)
    timed(ra, R.MODE_ATOMIC, R.PATH_PERSISTENT, 2)
    msa, eva, _ = timed(ra, R.MODE_ATOMIC, R.PATH_PERSISTENT, max(2, min(5, args.steps)))
    ra.release()
    ring_slots = (int(g.delays.max()) + 1) * g.num_neurons
    red_peak = R.probe_red_rate(ring_slots)
    red_ach = eva / (sum(msa) / 1e3)
    roofline["atomic"] = {"mode": "atomic", "achieved": red_ach, "peak": red_peak, "unit": "reductions/s",
                          "frac": red_ach / red_peak, "ms_per_launch": sum(msa) / len(msa),
                          "reductions_per_launch": eva / len(msa),
                          "peak_kind": f"measured here: snc_b200_probe_red_rate over {ring_slots} floats "
                                       "(the ring's size), scattered addresses, all SMs"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_extra:
        cpu, ref_counts = cpu_baseline(g, ev, lif)
        extra["parity"] = parity_leg(dg, di, g, ev, lif, mode, timed_out,
                                     ref_counts if cpu["kind"] == "reference" else None)
        extra["configs"] = config_legs()
        extra["reference_gpu"] = reference_gpu_leg(g_c2=g)
        extra["graph_build"] = graph_build_leg(g, t_build)
        extra["bptt"] = bptt_leg()

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded graph and Poisson drive, snc_b200/workloads.py)",
                "config": {"workload": WORKLOAD, "path": "persistent", "mode": R.MODE_NAMES[mode],
                           "cuda_graph": used_graph, "l2": "flushed (256 MiB write) before each timed step",
                           "parallelism": f"replicas x{world}" if world > 1 else "single"},
                "sample_steps_per_s": world * 1000 * args.steps / (tot_ms_max / 1e3),
                "e2e": e2e, "gpu_launches": args.steps, "roofline": roofline,
                "cpu_baseline": cpu, "clocks": clk}
        line.update(extra)
        print(json.dumps(line), flush=True)
    run.release()
    di.release()
    dg.release()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.leg:
        legs = {"bptt": bptt_leg, "bptt-custom": lambda: bptt_leg(with_reference=False),
                "configs": config_legs, "reference-gpu": reference_gpu_leg,
                "c3": lambda: c3_leg("atomic" if args.mode == "atomic" else "sort"),
                "eprop": eprop_leg}
        print(json.dumps({args.leg: legs[args.leg]()}), flush=True)
        return 0
    if args.impl == "reference":
        return reference_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())
