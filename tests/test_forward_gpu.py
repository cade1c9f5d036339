"""Parity of the B200 forward kernels against the CPU oracle and the
reference fixtures, through the C ABI.

SORT delivery must reproduce the serial CPU backend bit for bit: spike
rasters, final membrane potentials, logits, spike and event counts.  ATOMIC
and BUCKET delivery reorder float additions, so they are held to total
spike-count agreement >= 99.9% (the north-star tolerance for atomic mode).
"""
import numpy as np
import pytest

from oracle import oracle as O
from snc_b200 import runtime as R
from snc_b200 import workloads as W
from snc_b200.graph import SNNGraph
from tests.helpers import golden, spike_count_agreement, to_lif

pytestmark = pytest.mark.gpu

PATHS = [("plain", R.PATH_PLAIN, False), ("tierS", R.PATH_PERSISTENT, False),
         ("tierG", R.PATH_PERSISTENT, True)]


def run_gpu(g, ev, steps, lif, mode, path, force_grid=False, cuda_graph=False, repeat=1):
    dg = R.DeviceGraph(g)
    di = R.DeviceInputs(dg, ev, steps)
    run = R.Run(dg, di, raster=True, vfinal=True, cuda_graph=cuda_graph, force_grid=force_grid)
    for _ in range(repeat):
        run.launch(lif, mode=mode, path=path)
        out = run.fetch(raster=True, vfinal=True)
    out["used"] = run.used()
    out["used_graph"] = run.used_graph()
    return out


def assert_exact(out, ref):
    np.testing.assert_array_equal(out["spikes"], ref["spikes"])
    np.testing.assert_array_equal(out["events"], ref["events"])
    np.testing.assert_array_equal(out["logits"], ref["logits"])
    np.testing.assert_array_equal(out["raster"], ref["raster"])
    np.testing.assert_array_equal(out["v"].view(np.uint32), ref["v"].view(np.uint32))


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("lifcfg", [(0, 1), (1, 0), (0, 2)])
@pytest.mark.parametrize("pname,path,force", PATHS)
def test_sort_bit_exact_random(seed, lifcfg, pname, path, force):
    reset_mode, refractory = lifcfg
    g = W.random_graph(seed, max_delay=2 + seed * 3)
    ev, steps = W.random_events(seed + 10, g, 4, [37, 5, 60, 0])
    lif = R.LIFParams(threshold=1.0, decay=0.9, reset=0.0, refractory=refractory,
                      reset_mode=reset_mode)
    ref = O.forward_batched(g, ev, steps, lif)
    out = run_gpu(g, ev, steps, lif, R.MODE_SORT, path, force_grid=force)
    assert_exact(out, ref)


@pytest.mark.parametrize("mode", [R.MODE_ATOMIC, R.MODE_BUCKET])
@pytest.mark.parametrize("pname,path,force", PATHS)
def test_unordered_modes_spike_agreement(mode, pname, path, force):
    g = W.random_graph(5, n_hid=200, max_delay=6)
    ev, steps = W.random_events(9, g, 6, 80)
    lif = R.LIFParams(threshold=1.0, decay=0.9, refractory=1)
    ref = O.forward_batched(g, ev, steps, lif)
    out = run_gpu(g, ev, steps, lif, mode, path, force_grid=force)
    assert spike_count_agreement(out["spikes"], ref["spikes"]) >= 0.999
    assert out["used"] == (mode, path)


@pytest.mark.parametrize("prefix", ["static", "rsparse", "sdelay"])
@pytest.mark.parametrize("pname,path,force", PATHS)
def test_reference_fixture(prefix, pname, path, force):
    """Outputs of the unchanged reference CPU backend (tests/golden)."""
    g, ev, steps, lifns, exp = golden(prefix)
    lif = to_lif(lifns)
    out = run_gpu(g, ev, steps, lif, R.MODE_SORT, path, force_grid=force)
    np.testing.assert_array_equal(out["spikes"], exp["spikes"])
    np.testing.assert_array_equal(out["events"], exp["events"])
    np.testing.assert_array_equal(out["logits"], exp["logits"])


def test_one_call_forward_matches_reference_fixture():
    """snc_b200_forward: the cuda::forward replacement (graph uploaded inside)."""
    g, ev, steps, lifns, exp = golden("static")
    lif = to_lif(lifns)
    for i in range(3):
        evi = ev[ev["sample_id"] == i]
        r = R.forward(g, evi, int(steps[i]), lif, backend="cuda-sort")
        np.testing.assert_array_equal(r.logits, exp["logits"][i])
        assert r.stats.spikes == exp["spikes"][i]
        assert r.stats.synaptic_events == exp["events"][i]
        assert r.used_backend == "b200-sort"


def test_ff784_persistent_vs_oracle():
    g = W.ff784_graph()
    ev, steps = W.ff784_inputs(64)
    lif = W.lif_tau20()
    ref = O.forward_batched(g, ev, steps, lif)
    out = run_gpu(g, ev, steps, lif, R.MODE_SORT, R.PATH_PERSISTENT, cuda_graph=True, repeat=2)
    assert_exact(out, ref)
    assert out["used_graph"]


def test_audio700_uneven_persistent_vs_oracle():
    g = W.audio700_graph()
    ev, steps = W.audio700_inputs(12)
    lif = W.lif_tau20()
    ref = O.forward_batched(g, ev, steps, lif)
    for force in (False, True):
        out = run_gpu(g, ev, steps, lif, R.MODE_SORT, R.PATH_PERSISTENT, force_grid=force)
        assert_exact(out, ref)


@pytest.fixture(scope="module")
def rec100k():
    g = W.rec100k_graph()
    ev, steps = W.rec100k_inputs(g, num_samples=2, num_steps=300)
    lif = W.lif_tau20()
    return g, ev, steps, lif, O.forward_batched(g, ev, steps, lif)


@pytest.mark.parametrize("path", [R.PATH_PLAIN, R.PATH_PERSISTENT])
def test_rec100k_sort_bit_exact(rec100k, path):
    g, ev, steps, lif, ref = rec100k
    out = run_gpu(g, ev, steps, lif, R.MODE_SORT, path, cuda_graph=(path == R.PATH_PERSISTENT))
    assert_exact(out, ref)


@pytest.mark.parametrize("mode", [R.MODE_ATOMIC, R.MODE_BUCKET])
def test_rec100k_unordered(rec100k, mode):
    g, ev, steps, lif, ref = rec100k
    out = run_gpu(g, ev, steps, lif, mode, R.PATH_PERSISTENT)
    assert spike_count_agreement(out["spikes"], ref["spikes"]) >= 0.999
    np.testing.assert_array_equal(out["events"].sum() > 0, True)


def test_empty_and_zero_step_inputs():
    g = W.random_graph(4)
    lif = R.LIFParams()
    out = run_gpu(g, None, [0, 3, 0], lif, R.MODE_SORT, R.PATH_PERSISTENT)
    ref = O.forward_batched(g, np.zeros(0, dtype=O.EVENT_DTYPE), [0, 3, 0], lif)
    assert_exact(out, ref)
    assert out["spikes"].sum() == 0


def test_batched_one_call_and_autotune():
    g = W.random_graph(6, n_hid=120)
    ev, steps = W.random_events(3, g, 5, [30, 40, 50, 20, 10])
    lif = R.LIFParams(refractory=1)
    ref = O.forward_batched(g, ev, steps, lif)
    dg = R.DeviceGraph(g)
    out = R.forward_batched(dg, ev, steps, lif, mode=R.MODE_SORT)
    np.testing.assert_array_equal(out["spikes"], ref["spikes"])
    np.testing.assert_array_equal(out["logits"], ref["logits"])
    di = R.DeviceInputs(dg, ev, steps)
    best = R.autotune(dg, di, lif)
    assert best["mode"] in (0, 1, 2) and best["path"] in (0, 1)
    run = R.Run(dg, di)
    run.launch(lif, mode=R.MODE_AUTO, path=R.PATH_AUTO)
    run.fetch()
    assert run.used() == (best["mode"], best["path"])


@pytest.mark.parametrize("pname,path,force", PATHS)
def test_sort_bit_exact_at_the_largest_delay(pname, path, force):
    # delays up to 255 (the backend's limit; 8 bits in the packed edge): a
    # 256-slot ring, slots that wrap many times over 600 steps
    g = W.random_graph(17, n_hid=90, max_delay=6)
    rng = np.random.default_rng(17)
    d = g.delays.copy()
    d[rng.random(d.shape[0]) < 0.3] = 255
    d[::7] = rng.integers(200, 256, d[::7].shape[0])
    g.delays = d.astype(np.int32)
    ev, steps = W.random_events(18, g, 3, [600, 300, 450], rate=0.3)
    lif = R.LIFParams(threshold=1.0, decay=0.95, reset=0.0, refractory=1, reset_mode=1)
    ref = O.forward_batched(g, ev, steps, lif)
    assert int(ref["spikes"].sum()) > 0
    out = run_gpu(g, ev, steps, lif, R.MODE_SORT, path, force_grid=force)
    assert_exact(out, ref)


@pytest.mark.parametrize("pname,path,force", PATHS)
def test_sort_bit_exact_hub_columns(pname, path, force):
    # 300 inputs onto 3 hidden neurons: hundreds of events reach one column in
    # one step, so the ordered apply runs its long-list forms (chunks above
    # the serial-link size, column lists longer than the register sort)
    g = W.random_graph(23, n_in=300, n_hid=3, n_out=2, p=0.9, max_delay=3, recurrent=False)
    ev, steps = W.random_events(24, g, 3, [40, 25, 33], rate=0.5)
    lif = R.LIFParams(threshold=1.0, decay=0.9, reset=0.0, refractory=0, reset_mode=1)
    ref = O.forward_batched(g, ev, steps, lif)
    assert int(ref["events"].sum()) > 20000
    out = run_gpu(g, ev, steps, lif, R.MODE_SORT, path, force_grid=force)
    assert_exact(out, ref)


@pytest.mark.parametrize("pname,path,force", PATHS)
def test_sort_bit_exact_when_an_inbox_overflows(pname, path, force):
    # 3000 inputs spread over the grid kernel's blocks all feed the few
    # hidden neurons of the last block: every step a thousand or more
    # descriptors reach one inbox, more than it takes, so that block orders
    # its events from every block's fired list (the scan fallback) while the
    # others publish their lists after their barrier arrival
    g = W.random_graph(31, n_in=3000, n_hid=8, n_out=2, p=0.6, max_delay=4, recurrent=False)
    ev, steps = W.random_events(32, g, 1, [30], rate=0.9)
    lif = R.LIFParams(threshold=0.5, decay=0.9, reset=0.0, refractory=0, reset_mode=1)
    ref = O.forward_batched(g, ev, steps, lif)
    assert int(ref["events"].sum()) > 20000
    out = run_gpu(g, ev, steps, lif, R.MODE_SORT, path, force_grid=force)
    assert_exact(out, ref)
    # the same twice more in one run object: stale fired counts from the
    # previous launch must not be taken for this one's
    out2 = run_gpu(g, ev, steps, lif, R.MODE_SORT, path, force_grid=force, repeat=2)
    assert_exact(out2, ref)


@pytest.mark.parametrize("pname,path,force", PATHS)
def test_graph_without_synapses(pname, path, force):
    # inputs fire from their drive alone; nothing is delivered
    N = 7
    role = np.array([1, 1, 1, 1, 0, 2, 2], np.uint8)
    channel = np.array([0, 1, 2, 2, -1, 0, 1], np.int32)
    g = SNNGraph(N, np.zeros(N + 1, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32),
                 np.zeros(0, np.int32), role, np.ones(N, np.int8), channel)
    ev, steps = W.random_events(31, g, 2, [20, 9], rate=0.6)
    lif = R.LIFParams(threshold=1.0, decay=0.9, refractory=1)
    ref = O.forward_batched(g, ev, steps, lif)
    assert int(ref["spikes"].sum()) > 0 and int(ref["events"].sum()) == 0
    out = run_gpu(g, ev, steps, lif, R.MODE_SORT, path, force_grid=force)
    assert_exact(out, ref)


# ---- the benchmarked configurations at their own sizes ---------------------

@pytest.fixture(scope="module")
def rec100k_bench():
    """The bench's headline input: rec100k seed 1, one sample of 1000 steps
    with Poisson drive seed 1, tau_mem 20 with subtractive reset."""
    g = W.rec100k_graph(seed=1)
    ev, steps = W.rec100k_inputs(g, 1, 1000, seed=1)
    lif = W.lif_tau20()
    return g, ev, steps, lif, O.forward_batched(g, ev, steps, lif)


@pytest.mark.parametrize("path,graph", [(R.PATH_PLAIN, False), (R.PATH_PERSISTENT, True),
                                        (R.PATH_PERSISTENT, False)])
def test_rec100k_bench_input_sort_bit_exact(rec100k_bench, path, graph):
    g, ev, steps, lif, ref = rec100k_bench
    out = run_gpu(g, ev, steps, lif, R.MODE_SORT, path, cuda_graph=graph, repeat=2)
    assert int(ref["spikes"].sum()) > 100_000
    assert_exact(out, ref)


@pytest.mark.parametrize("mode", [R.MODE_ATOMIC, R.MODE_BUCKET])
@pytest.mark.parametrize("path", [R.PATH_PLAIN, R.PATH_PERSISTENT])
def test_rec100k_bench_input_unordered(rec100k_bench, mode, path):
    g, ev, steps, lif, ref = rec100k_bench
    out = run_gpu(g, ev, steps, lif, mode, path, cuda_graph=(path == R.PATH_PERSISTENT))
    assert spike_count_agreement(out["spikes"], ref["spikes"]) >= 0.999
    assert spike_count_agreement(out["events"], ref["events"]) >= 0.999


@pytest.fixture(scope="module")
def audio700_all():
    g = W.audio700_graph()
    ev, steps = W.audio700_inputs(256)
    lif = W.lif_tau20()
    return g, ev, steps, lif, O.forward_batched(g, ev, steps, lif)


@pytest.mark.parametrize("path,force,graph", [(R.PATH_PERSISTENT, False, True),
                                              (R.PATH_PERSISTENT, True, False),
                                              (R.PATH_PLAIN, False, False)])
def test_audio700_all_256_samples_sort_bit_exact(audio700_all, path, force, graph):
    """C3 as benchmarked: all 256 uneven samples (50-1000 steps) in one
    launch, rasters and potentials bit-identical on every path."""
    g, ev, steps, lif, ref = audio700_all
    out = run_gpu(g, ev, steps, lif, R.MODE_SORT, path, force_grid=force, cuda_graph=graph)
    assert len(steps) == 256
    assert_exact(out, ref)


def test_audio700_all_256_samples_atomic(audio700_all):
    g, ev, steps, lif, ref = audio700_all
    out = run_gpu(g, ev, steps, lif, R.MODE_ATOMIC, R.PATH_PERSISTENT, cuda_graph=True)
    assert spike_count_agreement(out["spikes"], ref["spikes"]) >= 0.999


# ---- launch shapes and the autotuner ----------------------------------------

@pytest.mark.parametrize("shape", [dict(tier=0), dict(tier=1, block_threads=512, wave=1, ring_smem=1),
                                   dict(tier=1, block_threads=768, wave=2, ring_smem=0),
                                   dict(tier=1, block_threads=512, wave=0, ring_smem=0),
                                   dict(tier=1, block_threads=768, wave=3, ring_smem=1)])
@pytest.mark.parametrize("mode", [R.MODE_SORT, R.MODE_BUCKET, R.MODE_ATOMIC])
def test_every_launch_shape_keeps_the_results(shape, mode):
    g = W.random_graph(8, n_hid=400, max_delay=9)
    ev, steps = W.random_events(19, g, 5, [40, 12, 33, 0, 25])
    lif = R.LIFParams(threshold=1.0, decay=0.9, reset=0.0, refractory=1)
    ref = O.forward_batched(g, ev, steps, lif)
    dg = R.DeviceGraph(g)
    di = R.DeviceInputs(dg, ev, steps)
    run = R.Run(dg, di, raster=True, vfinal=True)
    run.configure(mode=mode, **shape)
    run.launch(lif, mode=mode, path=R.PATH_PERSISTENT)
    out = run.fetch(raster=True, vfinal=True)
    if mode == R.MODE_SORT:
        assert_exact(out, ref)
    else:
        assert spike_count_agreement(out["spikes"], ref["spikes"]) >= 0.999


def test_autotuner_times_launch_shapes_and_keys_on_the_graph():
    """The tuner times real launch shapes (tier-1 block sizes and ring
    placements beside the modes and paths), picks the fastest, AUTO launches
    use it, and a second graph of the same size but other contents is not
    covered by the first graph's entry."""
    lif = W.lif_tau20()
    g1 = W.rec100k_graph(seed=1, n=20000, width=200, out_degree=40)
    g2 = W.rec100k_graph(seed=2, n=20000, width=200, out_degree=40)
    assert (g1.num_neurons, g1.num_synapses) == (g2.num_neurons, g2.num_synapses)
    ev1, steps = W.rec100k_inputs(g1, 1, 300, seed=1)
    ev2, _ = W.rec100k_inputs(g2, 1, 300, seed=1)
    dg1, dg2 = R.DeviceGraph(g1), R.DeviceGraph(g2)
    di1, di2 = R.DeviceInputs(dg1, ev1, steps), R.DeviceInputs(dg2, ev2, steps)
    tuned = R.autotune(dg1, di1, lif)
    cands = tuned["candidates"]
    tier1 = [c for c in cands if c["path"] == R.PATH_PERSISTENT and c["tier"] == 1]
    assert len({c["block_threads"] for c in tier1}) >= 2
    assert {c["ring_smem"] for c in tier1 if c["mode"] != R.MODE_ATOMIC} == {0, 1}
    assert any(c["path"] == R.PATH_PLAIN for c in cands)
    assert len({c["ms"] for c in cands}) > 1
    assert tuned["ms"] == min(c["ms"] for c in cands)
    assert R.autotune_lookup(dg1, di1) == {k: v for k, v in tuned.items() if k != "candidates"}
    assert R.autotune_lookup(dg2, di2) is None
    run = R.Run(dg1, di1)
    run.launch(lif, mode=R.MODE_AUTO, path=R.PATH_AUTO)
    run.fetch()
    assert run.used() == (tuned["mode"], tuned["path"])


# ---- leaky readout units ------------------------------------------------------

@pytest.mark.parametrize("pname,path,force", PATHS)
@pytest.mark.parametrize("cuda_graph", [False, True])
def test_leaky_readout_units_bit_exact(pname, path, force, cuda_graph):
    """OUTPUT neurons as leaky readout units (ro_decay 0.9): logits (final
    potential / T, per channel), rasters and potentials bit-identical to the
    restatement on every path; switching them off restores spike counts."""
    g = W.random_graph(9, n_hid=150, n_out=6, max_delay=8)
    ev, steps = W.random_events(21, g, 4, [45, 0, 30, 60])
    lif = R.LIFParams(threshold=1.0, decay=0.9, reset=0.0, refractory=1, reset_mode=1)
    ref = O.forward_batched(g, ev, steps, lif, ro_decay=0.9)
    dg = R.DeviceGraph(g)
    di = R.DeviceInputs(dg, ev, steps)
    run = R.Run(dg, di, raster=True, vfinal=True, cuda_graph=cuda_graph, force_grid=force)
    run.set_readout(0.9)
    for _ in range(2):
        run.launch(lif, mode=R.MODE_SORT, path=path)
        out = run.fetch(raster=True, vfinal=True)
        assert_exact(out, ref)
    assert np.abs(ref["logits"]).sum() > 0
    run.set_readout(None)
    run.launch(lif, mode=R.MODE_SORT, path=path)
    assert_exact(run.fetch(raster=True, vfinal=True), O.forward_batched(g, ev, steps, lif))


def test_audio700_all_256_samples_leaky_readout(audio700_all):
    """C3 as configured: 20 leaky readout units (ro_decay 0.9) on all 256
    uneven samples in one graph-launched persistent run."""
    g, ev, steps, lif, _ = audio700_all
    ref = O.forward_batched(g, ev, steps, lif, ro_decay=0.9)
    dg = R.DeviceGraph(g)
    di = R.DeviceInputs(dg, ev, steps)
    run = R.Run(dg, di, raster=True, vfinal=True, cuda_graph=True)
    run.set_readout(0.9)
    run.launch(lif, mode=R.MODE_SORT, path=R.PATH_PERSISTENT)
    out = run.fetch(raster=True, vfinal=True)
    assert run.used_graph()
    assert_exact(out, ref)


# ---- post-neuron partitions ------------------------------------------------------

@pytest.mark.parametrize("world", [1, 2, 3])
def test_partitions_on_one_device_equal_the_single_run(world):
    """snc_b200_part_*: `world` partitions stepped in turn on one device with
    a shared spike-bit buffer reproduce the single-device run bit for bit."""
    from snc_b200 import parallel as PAR
    g = W.rec100k_graph(seed=3, n=20000, width=200, out_degree=40, max_delay=20)
    ev, steps = W.rec100k_inputs(g, 1, 300, rate=0.04, seed=3)
    lif = W.lif_tau20()
    ref = O.forward_batched(g, ev, steps, lif)
    dg = R.DeviceGraph(g)
    di = R.DeviceInputs(dg, ev, steps)
    outs = PAR.run_partitions_on_one_device(dg, di, lif, world)
    raster = np.bitwise_or.reduce([o["raster"] for o in outs])
    np.testing.assert_array_equal(raster, ref["raster"])
    v = np.concatenate([o["v"] for o in outs])
    np.testing.assert_array_equal(v.view(np.uint32), ref["v"][0].view(np.uint32))
    assert sum(o["spikes"] for o in outs) == int(ref["spikes"][0]) > 0
    assert sum(o["events"] for o in outs) == int(ref["events"][0])
    np.testing.assert_array_equal(np.sum([o["logits"] for o in outs], 0), ref["logits"][0])


def test_partitions_on_the_bench_input(rec100k_bench):
    """rec100k's benchmarked input (1000 steps) split over two partitions."""
    from snc_b200 import parallel as PAR
    g, ev, steps, lif, ref = rec100k_bench
    dg = R.DeviceGraph(g)
    di = R.DeviceInputs(dg, ev, steps)
    outs = PAR.run_partitions_on_one_device(dg, di, lif, 2)
    np.testing.assert_array_equal(np.bitwise_or.reduce([o["raster"] for o in outs]), ref["raster"])
    v = np.concatenate([o["v"] for o in outs])
    np.testing.assert_array_equal(v.view(np.uint32), ref["v"][0].view(np.uint32))
    assert sum(o["events"] for o in outs) == int(ref["events"][0])


@pytest.mark.parametrize("batch", [1, 4, 16, 40])
def test_atomic_small_and_uneven_batches(batch):
    """ATOMIC on batches from one sample to a few dozen with uneven lengths
    on a 4000-neuron recurrent graph: spike totals agree with the CPU
    backend (the unordered modes' bar), every sample's within 1 %, and the
    rasters stay close."""
    g = W.rec100k_graph(seed=6, n=4000, width=80, out_degree=40, long_range=2, max_delay=9)
    ev, steps = W.rec100k_inputs(g, batch, 60, rate=0.06, seed=3)
    steps = np.asarray(steps).copy()
    steps[::3] = np.maximum(1, steps[::3] // 2)  # uneven lengths
    ev = ev[ev["time"] < steps[ev["sample_id"]]]
    lif = W.lif_tau20()
    ref = O.forward_batched(g, ev, steps, lif)
    assert int(ref["spikes"].sum()) > 0
    out = run_gpu(g, ev, steps, lif, R.MODE_ATOMIC, R.PATH_PERSISTENT)
    assert spike_count_agreement(out["spikes"], ref["spikes"]) >= 0.999
    for b in range(batch):
        assert spike_count_agreement(out["spikes"][b], ref["spikes"][b]) >= 0.99
    agree = np.mean(out["raster"] == ref["raster"])
    assert agree >= 0.99


def test_one_call_forward_from_pinned_host_events():
    """The end-to-end call with its events in pinned host memory (the
    bench's e2e leg) equals the same call from pageable memory and the CPU
    backend."""
    import torch
    g = W.random_graph(12, n_hid=120, max_delay=7)
    ev, steps = W.random_events(13, g, 5, [40, 22, 40, 31, 9])
    lif = R.LIFParams(threshold=1.0, decay=0.9, reset=0.0, refractory=1)
    ref = O.forward_batched(g, ev, steps, lif)
    dg = R.DeviceGraph(g)
    pin = torch.empty(ev.nbytes, dtype=torch.uint8, pin_memory=True)
    ev_pinned = pin.numpy().view(ev.dtype)
    ev_pinned[:] = ev
    a = R.forward_batched(dg, ev_pinned, steps, lif, mode=R.MODE_SORT)
    b = R.forward_batched(dg, ev, steps, lif, mode=R.MODE_SORT)
    for k in ("spikes", "events", "logits"):
        np.testing.assert_array_equal(a[k], b[k])
        np.testing.assert_array_equal(a[k], ref[k])


def test_reduction_rate_probe():
    """The atomic roofline's denominator: a positive, plausible rate of
    scattered float reductions (well above a billion per second)."""
    rate = R.probe_red_rate(1 << 20, 1 << 24)
    assert 1e9 < rate < 1e13
