"""The custom BPTT kernels against the autograd restatement of the bridge
(oracle/bptt_ref.py, pinned to the reference's SNN / SHDNet in
tests/test_bptt_ref.py).

Forward spikes must be bit-identical (the incoming edges are summed in the
order of torch's CPU index_add with the same roundings); gradients agree
within 1e-4 relative to their largest magnitude; checkpointing with
recompute changes nothing; the smoothed variant matches finite differences.
"""
import numpy as np
import pytest
import torch

from oracle import bptt_ref as BR
from snc_b200 import bptt as BP
from snc_b200 import workloads as W

pytestmark = pytest.mark.gpu
DEV = "cuda"


def graph(seed, n_in=24, n_hid=70, n_out=6, max_delay=4):
    g = W.random_graph(seed, n_in=n_in, n_hid=n_hid, n_out=n_out, max_delay=max_delay, w_scale=0.8)
    rng = np.random.default_rng(seed)
    w = (rng.normal(0, 0.6, g.num_synapses) * np.where(rng.random(g.num_synapses) < 0.3, -1, 1)).astype(np.float32)
    return g, w


def ref_run(g, w, ext, thr, decay, k, proj, smooth=False, dtype=torch.float32):
    wt = torch.as_tensor(w, dtype=dtype).clone().requires_grad_(True)
    et = ext.to(dtype).clone().requires_grad_(True)
    s = BR.core_forward(wt, et, torch.as_tensor(g.pre_ids()).long(), torch.as_tensor(g.post_ids).long(),
                        torch.as_tensor(g.delays).long(), thr, decay, k, smooth=smooth)
    (s * proj.to(dtype)).sum().backward()
    return s.detach(), wt.grad, et.grad


def gpu_run(g, w, ext, thr, decay, k, proj, ckpt, smooth=False):
    core = BP.SpikingCore(g.num_neurons, g.pre_ids(), g.post_ids, g.delays, device=DEV)
    wt = torch.as_tensor(w, device=DEV).clone().requires_grad_(True)
    et = ext.to(DEV).clone().requires_grad_(True)
    s = BP.spiking_core(wt, et, core, thr, decay, k, ckpt, smooth)
    (s * proj.to(DEV)).sum().backward()
    return s.detach().cpu(), wt.grad.cpu(), et.grad.cpu()


def rel_close(a, b, tol=1e-4):
    scale = max(float(b.abs().max()), 1e-12)
    assert float((a - b).abs().max()) <= tol * scale, (float((a - b).abs().max()), scale)


@pytest.mark.parametrize("B", [5, 32, 40, 128])
@pytest.mark.parametrize("ckpt", [0, 3, 10])
def test_forward_exact_and_gradients(B, ckpt):
    g, w = graph(1)
    T = 23
    gen = torch.Generator().manual_seed(B)
    ext = (torch.rand(T, B, g.num_neurons, generator=gen) < 0.25).float() * 1.1
    ext[:, :, 24:] = 0.0
    proj = torch.randn(T, B, g.num_neurons, generator=gen)
    s_ref, gw_ref, ge_ref = ref_run(g, w, ext, 1.0, 0.9, 25.0, proj)
    s, gw, ge = gpu_run(g, w, ext, 1.0, 0.9, 25.0, proj, ckpt)
    assert s_ref.sum() > 0
    assert torch.equal(s, s_ref)
    rel_close(gw, gw_ref)
    rel_close(ge, ge_ref)


def test_checkpointing_is_exact():
    g, w = graph(2, max_delay=7)
    T, B = 31, 16
    gen = torch.Generator().manual_seed(0)
    ext = torch.rand(T, B, g.num_neurons, generator=gen) * 0.6
    proj = torch.randn(T, B, g.num_neurons, generator=gen)
    outs = [gpu_run(g, w, ext, 1.0, 0.95, 25.0, proj, k) for k in (0, 1, 4, 10, 64)]
    for o in outs[1:]:
        assert torch.equal(o[0], outs[0][0])
        assert torch.equal(o[1], outs[0][1])
        assert torch.equal(o[2], outs[0][2])


def test_smooth_variant_against_fp64_and_finite_differences():
    g, w = graph(3, n_hid=40, max_delay=3)
    w = (w * 0.5).astype(np.float32)
    T, B = 12, 8
    gen = torch.Generator().manual_seed(1)
    ext = torch.rand(T, B, g.num_neurons, generator=gen)
    proj = torch.randn(T, B, g.num_neurons, generator=gen)
    _, gw64, ge64 = ref_run(g, w, ext, 0.5, 0.9, 5.0, proj, smooth=True, dtype=torch.float64)
    _, gw, ge = gpu_run(g, w, ext, 0.5, 0.9, 5.0, proj, 4, smooth=True)
    rel_close(gw.double(), gw64, 1e-4)
    rel_close(ge.double(), ge64, 1e-4)
    core = BP.SpikingCore(g.num_neurons, g.pre_ids(), g.post_ids, g.delays, device=DEV)
    e_d, p_d = ext.to(DEV), proj.to(DEV)

    def loss(wv):
        with torch.no_grad():
            return float((BP.spiking_core(torch.as_tensor(wv, device=DEV), e_d, core, 0.5, 0.9, 5.0, 0,
                                          True) * p_d).double().sum())

    eps = 2e-3
    for i in np.random.default_rng(0).choice(g.num_synapses, 8, replace=False):
        wp, wm = w.copy(), w.copy()
        wp[i] += eps
        wm[i] -= eps
        fd = (loss(wp) - loss(wm)) / (2 * eps)
        assert abs(fd - float(gw[i])) <= 2e-2 * max(1.0, abs(fd)), (i, fd, float(gw[i]))


def test_snn_dropin_matches_restatement():
    """snc_b200.bptt.SNN with the bridge constructor, direct encoding."""
    g, w = graph(4)
    d = {"N": g.num_neurons, "S": g.num_synapses, "n_in": g.num_input_channels,
         "n_out": g.num_output_channels, "pre": g.pre_ids(), "post": g.post_ids, "delays": g.delays,
         "role": g.role.astype(np.int32), "channel": g.channel}
    net = BP.SNN(d, num_steps=15, thr=1.0, decay=0.9, encoder="direct", surrogate_scale=25.0).to(DEV)
    with torch.no_grad():
        net.w.copy_(torch.as_tensor(w))
    x = torch.rand(9, d["n_in"], generator=torch.Generator().manual_seed(5))
    logits = net(x.to(DEV))
    logits.square().sum().backward()
    ext = torch.zeros(15, 9, d["N"])
    ext[:, :, :d["n_in"]] = x
    wt = torch.as_tensor(w).clone().requires_grad_(True)
    s = BR.core_forward(wt, ext, torch.as_tensor(d["pre"]).long(), torch.as_tensor(d["post"]).long(),
                        torch.as_tensor(d["delays"]).long(), 1.0, 0.9, 25.0)
    out_ids = torch.as_tensor(np.nonzero(d["role"] == 2)[0]).long()
    ref = torch.zeros(9, d["n_out"]).index_add(1, torch.as_tensor(d["channel"])[out_ids].long(),
                                               s.sum(0)[:, out_ids])
    assert torch.equal(logits.detach().cpu(), ref.detach())
    ref.square().sum().backward()
    rel_close(net.w.grad.cpu(), wt.grad)


def test_spiking_lm_gradients():
    H, V, T, B = 96, 12, 20, 8
    rng = np.random.default_rng(6)
    pre = np.repeat(np.arange(H), 8)
    post = (pre + rng.integers(-6, 7, pre.shape[0])) % H
    dl = rng.integers(1, 9, pre.shape[0])
    torch.manual_seed(0)
    lm = BP.SpikingLM(V, H, pre, post, dl, w_scale=2.0).to(DEV)
    with torch.no_grad():
        lm.embed.weight.mul_(1.5)
    x = torch.as_tensor(rng.integers(0, V, (B, T)))
    logits = lm(x.to(DEV))
    loss = torch.nn.functional.cross_entropy(logits.reshape(-1, V), x.reshape(-1).to(DEV))
    loss.backward()
    # autograd restatement with the same parameters
    emb = lm.embed.weight.detach().cpu().clone().requires_grad_(True)
    wr = lm.w_rec.detach().cpu().clone().requires_grad_(True)
    ext = emb[x].transpose(0, 1)
    s = BR.core_forward(wr, ext, torch.as_tensor(pre).long(), torch.as_tensor(post).long(),
                        torch.as_tensor(dl).long(), 1.0, 0.95, 25.0)
    r = torch.zeros(B, H)
    rs = []
    for t in range(T):
        r = 0.9 * r + s[t]
        rs.append(r)
    lg = torch.nn.functional.linear(torch.stack(rs, 1), lm.readout.weight.detach().cpu(),
                                    lm.readout.bias.detach().cpu())
    l2 = torch.nn.functional.cross_entropy(lg.reshape(-1, V), x.reshape(-1))
    l2.backward()
    assert s.sum() > 0
    rel_close(lm.w_rec.grad.cpu(), wr.grad, 1e-4)
    rel_close(lm.embed.weight.grad.cpu(), emb.grad, 1e-4)


def test_leaky_scan_matches_the_step_loop():
    torch.manual_seed(3)
    x = torch.randn(37, 5, 29, device=DEV)
    y = BP.leaky_scan(x, 0.9)
    r = torch.zeros(5, 29, device=DEV)
    ref = []
    for t in range(37):
        r = 0.9 * r + x[t]
        ref.append(r)
    assert torch.equal(y, torch.stack(ref))  # same roundings as the loop
    xg = x.clone().requires_grad_(True)
    g = torch.randn_like(x)
    (BP.leaky_scan(xg, 0.9) * g).sum().backward()
    xr = x.clone().requires_grad_(True)
    r = torch.zeros(5, 29, device=DEV)
    out = []
    for t in range(37):
        r = 0.9 * r + xr[t]
        out.append(r)
    (torch.stack(out) * g).sum().backward()
    rel_close(xg.grad.cpu(), xr.grad.cpu(), 1e-6)


def test_delayed_snn_readout_and_gradients():
    d = W.random_graph(8, n_in=20, n_hid=60, n_out=6, max_delay=4)
    pre = d.pre_ids()
    ro_ids = np.nonzero(np.asarray(d.role) == 2)[0]
    net = BP.DelayedSNN(d.num_neurons, pre, d.post_ids, d.delays, 20, ro_ids, 3, thr=1.0,
                        decay=0.9, surrogate_scale=25.0, ckpt_every=0, seed=2).to(DEV)
    T, B = 24, 7
    x = (torch.rand(T, B, 20, generator=torch.Generator().manual_seed(4)) < 0.3).float()
    F = torch.nn.functional
    y = torch.as_tensor(np.random.default_rng(1).integers(0, 3, B))
    F.cross_entropy(net(x.to(DEV)), y.to(DEV)).backward()
    wt = net.w.detach().cpu().clone().requires_grad_(True)
    wro = net.readout.weight.detach().cpu().clone().requires_grad_(True)
    bro = net.readout.bias.detach().cpu().clone().requires_grad_(True)
    ext = torch.zeros(T, B, d.num_neurons)
    ext[:, :, :20] = x
    s = BR.core_forward(wt, ext, torch.as_tensor(pre).long(), torch.as_tensor(d.post_ids).long(),
                        torch.as_tensor(d.delays).long(), 1.0, 0.9, 25.0)
    F.cross_entropy(BR.leaky_readout(s, wro, bro, torch.as_tensor(ro_ids).long(), 0.9), y).backward()
    assert s.sum() > 0
    rel_close(net.w.grad.cpu(), wt.grad, 1e-4)
    rel_close(net.readout.weight.grad.cpu(), wro.grad, 1e-4)
    rel_close(net.readout.bias.grad.cpu(), bro.grad, 1e-4)


def _run_core(g, w, ext, proj, ckpt, smooth, resident):
    core = BP.SpikingCore(g.num_neurons, g.pre_ids(), g.post_ids, g.delays, device=DEV)
    core.set_resident(resident)
    wt = torch.as_tensor(w, device=DEV).clone().requires_grad_(True)
    et = ext.to(DEV).clone().requires_grad_(True)
    s = BP.spiking_core(wt, et, core, 1.0, 0.9, 8.0, ckpt, smooth)
    (s * proj.to(DEV)).sum().backward()
    return s.detach().cpu(), wt.grad.cpu(), et.grad.cpu()


@pytest.mark.parametrize("smooth", [False, True])
@pytest.mark.parametrize("ckpt", [0, 4])
def test_resident_launch_is_bit_identical(smooth, ckpt):
    # edges staged in shared memory per warp against the global-memory form
    g, w = graph(7, n_hid=90)
    T, B = 19, 40
    gen = torch.Generator().manual_seed(3)
    ext = (torch.rand(T, B, g.num_neurons, generator=gen) < 0.3).float() * 1.2
    proj = torch.randn(T, B, g.num_neurons, generator=gen)
    a = _run_core(g, w, ext, proj, ckpt, smooth, True)
    b = _run_core(g, w, ext, proj, ckpt, smooth, False)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.numpy().view(np.uint32), y.numpy().view(np.uint32))


def test_hub_neuron_beyond_the_resident_limit():
    # one neuron with 300 outgoing and one with 300 incoming synapses: the
    # launch falls back to the global-memory form; still exact / within 1e-4
    rng = np.random.default_rng(5)
    N = 340
    pre = np.concatenate([np.zeros(300, np.int64), rng.integers(1, N, 300), rng.integers(0, N, 600)])
    post = np.concatenate([rng.integers(1, N, 300), np.full(300, 5), rng.integers(0, N, 600)])
    d = rng.integers(1, 4, pre.shape[0])
    from snc_b200.graph import from_edges
    role = np.zeros(N, np.uint8)
    g = from_edges(N, pre, post, np.ones(pre.shape[0], np.float32), d, role)
    w = (rng.normal(0, 0.3, g.num_synapses)).astype(np.float32)
    T, B = 12, 33
    gen = torch.Generator().manual_seed(9)
    ext = (torch.rand(T, B, N, generator=gen) < 0.3).float() * 1.1
    proj = torch.randn(T, B, N, generator=gen)
    s, gw, ge = gpu_run(g, w, ext, 1.0, 0.9, 8.0, proj, 4)
    rs, rgw, rge = ref_run(g, w, ext, 1.0, 0.9, 8.0, proj)
    np.testing.assert_array_equal(s.numpy(), rs.numpy())
    rel_close(gw, rgw)
    rel_close(ge, rge)


def test_layout_transpose_matches_torch():
    # the tiled layout change around the kernels, on a contiguous tensor, a
    # [B, T, N] tensor seen as [T, B, N], and ragged tile edges
    gen = torch.Generator().manual_seed(11)
    x = torch.randn(7, 45, 70, generator=gen).to(DEV)
    np.testing.assert_array_equal(BP._to_tnb(x).cpu().numpy(), x.permute(0, 2, 1).contiguous().cpu().numpy())
    y = torch.randn(45, 7, 70, generator=gen).to(DEV).transpose(0, 1)
    np.testing.assert_array_equal(BP._to_tnb(y).cpu().numpy(), y.permute(0, 2, 1).contiguous().cpu().numpy())
    z = torch.randn(5, 33, 129, generator=gen).to(DEV)
    np.testing.assert_array_equal(BP._from_tnb(z).cpu().numpy(), z.permute(0, 2, 1).contiguous().cpu().numpy())


def _grad_errors(g, r):
    """(largest |g - r| over the largest |r|, largest elementwise |g - r| / |r|
    over the entries with |r| >= 1e-2 of the largest)."""
    scale = float(r.abs().max())
    maxnorm = float((g - r).abs().max()) / max(scale, 1e-30)
    big = r.abs() >= 1e-2 * scale
    elem = float(((g - r).abs()[big] / r.abs()[big]).max()) if bool(big.any()) else 0.0
    return maxnorm, elem


def _bench_shape_case(pre, post, delays, N, w, ext, ckpt, seed):
    """Core spikes and weight / drive gradients of the custom kernels against
    the CPU autograd restatement on the same weights and drive."""
    gen = torch.Generator().manual_seed(seed)
    proj = torch.randn(ext.shape, generator=gen)
    wt = w.clone().requires_grad_(True)
    et = ext.clone().requires_grad_(True)
    s_ref = BR.core_forward(wt, et, torch.as_tensor(pre).long(), torch.as_tensor(post).long(),
                            torch.as_tensor(delays).long(), 1.0, 0.95, 25.0)
    (s_ref * proj).sum().backward()
    core = BP.SpikingCore(N, np.asarray(pre), np.asarray(post), np.asarray(delays), device=DEV)
    wg = w.to(DEV).clone().requires_grad_(True)
    eg = ext.to(DEV).clone().requires_grad_(True)
    s = BP.spiking_core(wg, eg, core, 1.0, 0.95, 25.0, ckpt, False)
    (s * proj.to(DEV)).sum().backward()
    assert float(s_ref.sum()) > 0
    assert torch.equal(s.detach().cpu(), s_ref.detach())
    return _grad_errors(wg.grad.cpu(), wt.grad), _grad_errors(eg.grad.cpu(), et.grad)


def test_mnist_like_bench_shape_gradients():
    """The benchmark's mnist-like BPTT configuration (784 Poisson -> 512 ->
    512 LIF, local sparse, delays 1-4, batch 128, checkpoints every 10 steps)
    with its own graph, weights and input spikes, T cut from 100 to 50 so the
    CPU autograd model stays small: forward spikes identical; weight and
    drive gradients within 1e-4, both relative to the largest gradient and
    elementwise over entries of at least 1e-2 of the largest."""
    c4 = W.bptt_mnist_like(T=50)
    model = BP.DelayedSNN(c4["N"], c4["pre"], c4["post"], c4["delays"], c4["n_in"],
                          c4["readout_ids"], 10, thr=1.0, decay=0.95, surrogate_scale=25.0,
                          ckpt_every=10)
    T, B = c4["spikes"].shape[:2]
    assert B == 128
    ext = torch.zeros(T, B, c4["N"])
    ext[:, :, :c4["n_in"]] = torch.as_tensor(c4["spikes"])
    (gw_max, gw_el), (ge_max, ge_el) = _bench_shape_case(c4["pre"], c4["post"], c4["delays"], c4["N"],
                                                         model.w.detach(), ext, 10, 4)
    assert gw_max <= 1e-4 and gw_el <= 1e-4, (gw_max, gw_el)
    assert ge_max <= 1e-4 and ge_el <= 1e-4, (ge_max, ge_el)


def test_char_lm_bench_shape_gradients():
    """The benchmark's char-LM configuration (4096 recurrent LIF, fan-in 64,
    delays 1-8, batch 64, checkpoints every 16 steps) with its own graph,
    weights and embedded Zipf tokens, T cut from 256 to 48: the same bars as
    the mnist-like case."""
    c5 = W.char_lm(T=48)
    torch.manual_seed(0)
    net = BP.SpikingLM(c5["vocab"], c5["H"], c5["pre"], c5["post"], c5["delays"], w_scale=2.0,
                       ckpt_every=16)
    with torch.no_grad():
        ext = net.embed(torch.as_tensor(c5["x"])).transpose(0, 1).contiguous()
    assert ext.shape[1] == 64
    (gw_max, gw_el), (ge_max, ge_el) = _bench_shape_case(c5["pre"], c5["post"], c5["delays"], c5["H"],
                                                         net.w_rec.detach(), ext, 16, 5)
    assert gw_max <= 1e-4 and gw_el <= 1e-4, (gw_max, gw_el)
    assert ge_max <= 1e-4 and ge_el <= 1e-4, (ge_max, ge_el)


def test_shard_gradients_add_up_to_the_full_batch():
    """Sample-sharded BPTT (snc_b200.parallel.shard_gradient, the per-rank
    half of DataParallelBPTT) with the custom kernels: the shards' gradients
    of the summed loss over 2 and 3 uneven shards add up to the whole batch's
    gradient (samples are independent; only the dW summation order across
    the batch differs)."""
    from snc_b200 import parallel as PAR
    d = W.random_graph(8, n_in=20, n_hid=60, n_out=6, max_delay=4)
    ro_ids = np.nonzero(np.asarray(d.role) == 2)[0]
    net = BP.DelayedSNN(d.num_neurons, d.pre_ids(), d.post_ids, d.delays, 20, ro_ids, 3, thr=1.0,
                        decay=0.9, surrogate_scale=25.0, ckpt_every=6, seed=2).to(DEV)
    T, B = 24, 7
    x = (torch.rand(T, B, 20, generator=torch.Generator().manual_seed(4)) < 0.3).float().to(DEV)
    y = torch.as_tensor(np.random.default_rng(1).integers(0, 3, B)).to(DEV)

    def loss_fn(m, xs, ys):
        return torch.nn.functional.cross_entropy(m(xs), ys, reduction="sum")

    full, lf = PAR.shard_gradient(net, loss_fn, x, y, 1, 0, 1)
    assert float(full.abs().max()) > 0
    for world in (2, 3):
        parts = [PAR.shard_gradient(net, loss_fn, x, y, 1, r, world) for r in range(world)]
        rel_close(sum(g for g, _ in parts).cpu(), full.cpu(), 1e-5)
        assert abs(float(sum(l for _, l in parts)) - float(lf)) <= 1e-5 * abs(float(lf))
