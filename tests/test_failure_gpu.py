"""Failure detection without a GPU fault.

* A bounded device wait that runs out: snc_b200_inject_stall makes the grid
  barriers of the next launch wait for an arrival that no block makes (a
  flag nothing sets); with a 10 ms wait limit every block gives up, the call
  reports SNC_B200_ETIMEOUT, and the next launch on the same context is
  bit-exact again.  Covers the all-SM forward (direct and CUDA-graph runs)
  and the BPTT forward / backward.
* A device allocation that fails on the host (snc_b200_inject_alloc_failure,
  SNC_B200_FAIL_ALLOC): the call returns SNC_B200_ENOMEM and nothing is left
  half-built; the reference's snc_bench linked with the adapter then takes
  its own CPU fallback (cpu_backend.cpp:197-205) and prints "(fallback)"
  with the cpu backend's counts.
"""
import os
import subprocess

import numpy as np
import pytest
import torch

from oracle import oracle as O
from snc_b200 import _lib
from snc_b200 import bptt as BP
from snc_b200 import runtime as R
from snc_b200 import workloads as W
from tests.test_forward_gpu import assert_exact

pytestmark = pytest.mark.gpu
LIMIT_NS = 10_000_000  # 10 ms


@pytest.fixture
def short_waits():
    L = _lib.lib()
    _lib.check(L.snc_b200_set_wait_limit(LIMIT_NS), "set_wait_limit")
    yield L
    L.snc_b200_inject_stall(0)
    L.snc_b200_set_wait_limit(0)


@pytest.mark.parametrize("mode", [R.MODE_SORT, R.MODE_BUCKET, R.MODE_ATOMIC])
@pytest.mark.parametrize("cuda_graph", [False, True])
def test_grid_wait_runs_out_and_the_context_recovers(short_waits, mode, cuda_graph):
    L = short_waits
    g = W.random_graph(5, n_hid=300, max_delay=7)
    ev, steps = W.random_events(15, g, 3, [40, 25, 60])
    lif = R.LIFParams(threshold=1.0, decay=0.9, reset=0.0, refractory=1)
    ref = O.forward_batched(g, ev, steps, lif)
    dg = R.DeviceGraph(g)
    di = R.DeviceInputs(dg, ev, steps)
    run = R.Run(dg, di, raster=True, vfinal=True, cuda_graph=cuda_graph, force_grid=True)
    if cuda_graph:  # a captured graph exists before the stalled launch
        run.launch(lif, mode=R.MODE_SORT, path=R.PATH_PERSISTENT)
        run.fetch()
    _lib.check(L.snc_b200_inject_stall(1), "inject_stall")
    run.launch(lif, mode=mode, path=R.PATH_PERSISTENT)
    with pytest.raises(_lib.SncB200Error) as ei:
        run.fetch()
    assert ei.value.status == _lib.ETIMEOUT
    assert "timed out" in str(ei.value)
    # the next launch runs normally on the same context
    run.launch(lif, mode=R.MODE_SORT, path=R.PATH_PERSISTENT)
    out = run.fetch(raster=True, vfinal=True)
    assert run.used_graph() == cuda_graph
    assert_exact(out, ref)


def test_bptt_wait_runs_out_and_the_next_call_is_unchanged(short_waits):
    L = short_waits
    g = W.random_graph(6, n_in=20, n_hid=90, n_out=5, max_delay=4, w_scale=0.8)
    core = BP.SpikingCore(g.num_neurons, g.pre_ids(), g.post_ids, g.delays, device="cuda")
    gen = torch.Generator().manual_seed(2)
    w = (torch.randn(g.num_synapses, generator=gen) * 0.6).cuda()
    T, B = 17, 24
    ext = (torch.rand(T, B, g.num_neurons, generator=gen) * 0.8).cuda()
    proj = torch.randn(T, B, g.num_neurons, generator=gen).cuda()

    def step():
        wt = w.clone().requires_grad_(True)
        s = BP.spiking_core(wt, ext, core, 1.0, 0.9, 25.0, 4, False)
        (s * proj).sum().backward()
        return s.detach().cpu(), wt.grad.cpu()

    s0, g0 = step()
    _lib.check(L.snc_b200_inject_stall(1), "inject_stall")
    with pytest.raises(_lib.SncB200Error) as ei:  # the forward's barriers give up
        step()
    assert ei.value.status == _lib.ETIMEOUT
    s1, g1 = step()
    assert torch.equal(s0, s1) and torch.equal(g0, g1)
    # a stall in the backward: the forward passes, the backward gives up
    wt = w.clone().requires_grad_(True)
    s = BP.spiking_core(wt, ext, core, 1.0, 0.9, 25.0, 4, False)
    _lib.check(L.snc_b200_inject_stall(1), "inject_stall")
    with pytest.raises(_lib.SncB200Error) as ei:
        (s * proj).sum().backward()
    assert ei.value.status == _lib.ETIMEOUT
    s2, g2 = step()
    assert torch.equal(s0, s2) and torch.equal(g0, g2)


def test_failed_allocation_is_reported_and_recovers():
    L = _lib.lib()
    g = W.random_graph(7)
    ev, steps = W.random_events(17, g, 2, [30, 20])
    lif = R.LIFParams()
    try:
        for allowed in (0, 3):
            _lib.check(L.snc_b200_inject_alloc_failure(allowed), "inject_alloc_failure")
            with pytest.raises(_lib.SncB200Error) as ei:
                R.DeviceGraph(g)
            assert ei.value.status == _lib.ENOMEM
            assert "injected" in str(ei.value)
    finally:
        L.snc_b200_inject_alloc_failure(-1)
    dg = R.DeviceGraph(g)
    di = R.DeviceInputs(dg, ev, steps)
    run = R.Run(dg, di, raster=True, vfinal=True)
    run.launch(lif, mode=R.MODE_SORT, path=R.PATH_PERSISTENT)
    assert_exact(run.fetch(raster=True, vfinal=True), O.forward_batched(g, ev, steps, lif))


def test_reference_cli_takes_its_cpu_fallback_when_the_device_path_fails():
    """snc::forward (cpu_backend.cpp:197-205): cuda::forward returning false
    makes the reference run its CPU backend and report used_backend = cpu."""
    bench = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "snc_b200",
                         "adapter", "_build", "snc_bench")
    if not os.path.exists(bench):
        pytest.skip("reference CLIs not built")
    args = [bench, "--structure", "static-snc", "--num-steps", "30", "--num-samples", "8",
            "--hidden", "128", "--compare-backends"]
    env = dict(os.environ, SNC_B200_FAIL_ALLOC="0")
    out = subprocess.run(args, capture_output=True, text=True, timeout=300, env=env)
    assert out.returncode == 0, out.stderr
    lines = [l for l in out.stdout.splitlines() if l.strip()]
    cpu = [l.split() for l in lines if l.startswith("cpu ")][0]
    fallback = [l.split() for l in lines if "(fallback)" in l]
    assert len(fallback) == 3, out.stdout  # cuda-atomic, cuda-bucket, cuda-sort
    for f in fallback:
        assert f[0] == "cpu" and f[1:3] == cpu[1:3] and f[5] == "exact", out.stdout
    ok = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert ok.returncode == 0 and "(fallback)" not in ok.stdout, ok.stdout
