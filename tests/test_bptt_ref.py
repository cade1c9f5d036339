"""The BPTT autograd restatement (oracle/bptt_ref.py) pinned against the
reference bridge's own modules where the reference tree is present
(python/snc/model.py SNN for delay-1 graphs, python/snc/shd_model.py SHDNet
for per-synapse delays), and against finite differences of its smoothed
variant."""
import importlib.util
import os
import sys

import numpy as np
import pytest
import torch

from oracle import REF_ROOT
from oracle import bptt_ref as BR
from snc_b200 import workloads as W

REF_PY = os.path.join(REF_ROOT, "python")
needs_ref_py = pytest.mark.skipif(not os.path.isdir(os.path.join(REF_PY, "snc")),
                                  reason="reference python bridge absent")


def _ref_snc():
    if REF_PY not in sys.path:
        sys.path.insert(0, REF_PY)
    import snc.model as model  # noqa: E402
    import snc.shd_model as shd  # noqa: E402
    return model, shd


def graph_dict(g):
    return {"N": g.num_neurons, "S": g.num_synapses, "n_in": g.num_input_channels,
            "n_out": g.num_output_channels, "pre": g.pre_ids(), "post": g.post_ids,
            "delays": g.delays, "role": g.role.astype(np.int32), "channel": g.channel}


@needs_ref_py
def test_matches_reference_snn_delay1():
    model, _ = _ref_snc()
    g = W.random_graph(3, n_in=16, n_hid=40, n_out=4, max_delay=1, recurrent=False)
    g.delays[:] = 1
    d = graph_dict(g)
    net = model.SNN(d, num_steps=12, thr=1.0, decay=0.9, gain=1.0, encoder="direct",
                    surrogate_scale=25.0, seed=2)
    # the reference drives input neurons 0..dim-1 with x * gain every step
    x = torch.rand(5, d["n_in"], generator=torch.Generator().manual_seed(0)) * 1.2
    out_ref = net(x)
    loss_ref = (out_ref * torch.arange(1, d["n_out"] + 1)).sum()
    loss_ref.backward()
    w = net.w.detach().clone().requires_grad_(True)
    ext = torch.zeros(12, 5, d["N"])
    ext[:, :, :d["n_in"]] = x
    s = BR.core_forward(w, ext, torch.as_tensor(d["pre"]).long(), torch.as_tensor(d["post"]).long(),
                        torch.as_tensor(d["delays"]).long(), 1.0, 0.9, 25.0)
    out_ids = torch.as_tensor(np.nonzero(d["role"] == 2)[0]).long()
    out = torch.zeros(5, d["n_out"]).index_add(1, torch.as_tensor(d["channel"][out_ids.numpy()]).long(),
                                               s.sum(0)[:, out_ids])
    torch.testing.assert_close(out, out_ref.detach(), rtol=0, atol=0)
    (out * torch.arange(1, d["n_out"] + 1)).sum().backward()
    torch.testing.assert_close(w.grad, net.w.grad, rtol=1e-6, atol=1e-7)


@needs_ref_py
def test_matches_reference_shdnet_delays():
    _, shd = _ref_snc()
    H, n_in, C, T, B = 48, 20, 5, 30, 4
    rng = np.random.default_rng(4)
    a, b = np.nonzero(rng.random((H, H)) < 0.15)
    rp, rq = torch.as_tensor(a).long(), torch.as_tensor(b).long()
    rdel = torch.as_tensor(rng.integers(1, 6, a.shape[0])).long()
    a2, b2 = np.nonzero(rng.random((n_in, H)) < 0.3)
    ip, iq = torch.as_tensor(a2).long(), torch.as_tensor(b2).long()
    net = shd.SHDNet(n_in, [H], C, [(rp, rq)], rec_delays=[rdel], in_edges=(ip, iq), decay=0.95,
                     thr=1.0, surrogate_scale=25.0, w_rec_scale=1.5, seed=1, adaptive=False,
                     learn_tau=False, readout="leaky", ro_decay=0.9)
    x = (torch.rand(B, T, n_in, generator=torch.Generator().manual_seed(3)) < 0.3).float()
    y = net(x)
    y.square().sum().backward()
    w_rec = net.w_rec[0].detach().clone().requires_grad_(True)
    w_in = net.w_in.detach().clone().requires_grad_(True)
    w_ro = net.readout.weight.detach().clone().requires_grad_(True)
    b_ro = net.readout.bias.detach().clone().requires_grad_(True)
    ext = torch.stack([torch.zeros(B, H).index_add(1, iq, w_in.unsqueeze(0) * x[:, t][:, ip])
                       for t in range(T)])
    s = BR.core_forward(w_rec, ext, rp, rq, rdel, 1.0, 0.95, 25.0)
    y2 = BR.leaky_readout(s, w_ro, b_ro, torch.arange(H), 0.9)
    torch.testing.assert_close(y2, y.detach(), rtol=1e-5, atol=1e-6)
    y2.square().sum().backward()
    torch.testing.assert_close(w_rec.grad, net.w_rec[0].grad, rtol=1e-4, atol=1e-6)
    torch.testing.assert_close(w_in.grad, net.w_in.grad, rtol=1e-4, atol=1e-6)
    torch.testing.assert_close(w_ro.grad, net.readout.weight.grad, rtol=1e-4, atol=1e-6)


def test_smooth_variant_finite_differences():
    """With s = x / (1 + k|x|) the surrogate is the exact derivative; the
    autograd gradient of the restatement must match central differences."""
    g = W.random_graph(2, n_in=8, n_hid=20, n_out=3, max_delay=4)
    T, B = 10, 3
    pre = torch.as_tensor(g.pre_ids()).long()
    post = torch.as_tensor(g.post_ids).long()
    dl = torch.as_tensor(g.delays).long()
    w = torch.as_tensor(g.weights, dtype=torch.float64).clone().requires_grad_(True)
    ext = torch.rand(T, B, g.num_neurons, dtype=torch.float64, generator=torch.Generator().manual_seed(1))
    proj = torch.randn(T, B, g.num_neurons, dtype=torch.float64, generator=torch.Generator().manual_seed(2))

    def loss(wv):
        return (BR.core_forward(wv, ext, pre, post, dl, 0.5, 0.9, 5.0, smooth=True) * proj).sum()

    loss(w).backward()
    eps = 1e-6
    idx = np.random.default_rng(0).choice(g.num_synapses, 12, replace=False)
    for i in idx:
        wp, wm = w.detach().clone(), w.detach().clone()
        wp[i] += eps
        wm[i] -= eps
        fd = (loss(wp) - loss(wm)).item() / (2 * eps)
        assert abs(fd - w.grad[i].item()) <= 1e-6 + 1e-5 * abs(fd)
