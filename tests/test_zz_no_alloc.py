"""snc_b200_bptt_forward_static -- the BPTT forward for callers that cannot
allocate device memory while they run it (a framework whose caching allocator
owns all device memory, a real-time loop that must not pay for or risk a
cudaMalloc) -- against the regular snc_b200_bptt_forward, through the C ABI,
on two calls in a row with different inputs (the second call must not see
the first call's leftovers in the shared static scratch).  Spikes, spike bits
and saved potentials must be identical.  A call on a fresh handle must leave
the device's free memory unchanged.

This file sorts last so that a run stopping at its first failure has already
run every other test; it also passes on its own in a fresh process."""
import ctypes as C

import numpy as np
import pytest
import torch

from snc_b200 import _lib
from snc_b200 import bptt as BP
from snc_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _call(fn_name, core, w, ext_t, T, B, K, smooth):
    N = core.N
    dev = ext_t.device
    spikes = torch.empty(T, N, B, device=dev)
    bits = torch.empty(T, N, (B + 31) // 32, device=dev, dtype=torch.int32)
    vsaved = torch.empty((T + K - 1) // K if K else T, N, B, device=dev)
    fn = getattr(_lib.lib(), fn_name)
    rc = fn(core.h, C.c_void_p(w.data_ptr()), C.c_void_p(ext_t.data_ptr()), T, B, 1.0, 0.9, 25.0, K,
            smooth, C.c_void_p(spikes.data_ptr()), C.c_void_p(bits.data_ptr()),
            C.c_void_p(vsaved.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc, fn_name)
    torch.cuda.synchronize()
    return spikes.cpu(), bits.cpu(), vsaved.cpu()


@pytest.mark.parametrize("K", [0, 4])
def test_static_forward_matches_regular_twice(K):
    _lib.check(_lib.lib().snc_b200_set_device(0), "set_device")
    g = W.random_graph(21, n_in=30, n_hid=120, n_out=8, max_delay=6, w_scale=0.8)
    core = BP.SpikingCore(g.num_neurons, g.pre_ids(), g.post_ids, g.delays, device="cuda")
    rng = np.random.default_rng(7)
    T, B = 25, 40
    w = torch.as_tensor(rng.normal(0, 0.6, g.num_synapses).astype(np.float32)[core.perm],
                        device="cuda")
    for call in range(2):
        ext = (torch.rand(T, g.num_neurons, B, generator=torch.Generator().manual_seed(call)) *
               (0.9 + 0.4 * call)).cuda()
        ref = _call("snc_b200_bptt_forward", core, w, ext, T, B, K, 0)
        got = _call("snc_b200_bptt_forward_static", core, w, ext, T, B, K, 0)
        assert ref[0].sum() > 0
        for a, b in zip(got, ref):
            assert torch.equal(a, b), f"call {call}: static forward differs"


def test_static_forward_rejects_oversize():
    g = W.random_graph(22, n_hid=40)
    core = BP.SpikingCore(g.num_neurons, g.pre_ids(), g.post_ids, g.delays, device="cuda")
    B = 1 + (1048512 // g.num_neurons)
    T = 1
    w = torch.zeros(g.num_synapses, device="cuda")
    ext = torch.zeros(T, g.num_neurons, 1, device="cuda")
    f = _lib.lib().snc_b200_bptt_forward_static
    dummy = torch.zeros(4, device="cuda")
    rc = f(core.h, C.c_void_p(w.data_ptr()), C.c_void_p(ext.data_ptr()), T, B, 1.0, 0.9, 25.0, 0, 0,
           C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()),
           None)
    assert rc == _lib.EUNSUPPORTED
    assert "static scratch" in _lib.lib().snc_b200_last_error().decode()


def test_static_forward_allocates_nothing():
    """A fresh handle (the regular forward never grew its state buffer): the
    static call leaves the device's free memory as it was.  The kernel is
    loaded by a first call on another handle, since loading code is the
    driver's doing, not the call's."""
    _lib.check(_lib.lib().snc_b200_set_device(0), "set_device")
    g = W.random_graph(23, n_in=30, n_hid=150, n_out=8, max_delay=5, w_scale=0.8)
    T, B = 20, 64
    w = torch.as_tensor(np.random.default_rng(3).normal(0, 0.6, g.num_synapses).astype(np.float32),
                        device="cuda")
    ext = torch.rand(T, g.num_neurons, B, generator=torch.Generator().manual_seed(5)).cuda()
    warm = BP.SpikingCore(g.num_neurons, g.pre_ids(), g.post_ids, g.delays, device="cuda")
    ref = _call("snc_b200_bptt_forward_static", warm, w[warm.perm_t].contiguous(), ext, T, B, 0, 0)
    fresh = BP.SpikingCore(g.num_neurons, g.pre_ids(), g.post_ids, g.delays, device="cuda")
    wf = w[fresh.perm_t].contiguous()
    N = fresh.N
    spikes = torch.empty(T, N, B, device="cuda")
    bits = torch.empty(T, N, (B + 31) // 32, device="cuda", dtype=torch.int32)
    vsaved = torch.empty(T, N, B, device="cuda")
    f = _lib.lib().snc_b200_bptt_forward_static
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    rc = f(fresh.h, C.c_void_p(wf.data_ptr()), C.c_void_p(ext.data_ptr()), T, B, 1.0, 0.9, 25.0, 0, 0,
           C.c_void_p(spikes.data_ptr()), C.c_void_p(bits.data_ptr()), C.c_void_p(vsaved.data_ptr()),
           C.c_void_p(torch.cuda.current_stream().cuda_stream))
    _lib.check(rc, "snc_b200_bptt_forward_static")
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    assert ref[0].sum() > 0
    assert torch.equal(spikes.cpu(), ref[0]) and torch.equal(bits.cpu(), ref[1])
