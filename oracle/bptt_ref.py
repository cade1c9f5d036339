"""PyTorch-autograd restatement of the reference bridge's surrogate-gradient
BPTT, generalised to per-synapse delays.  TEST INFRASTRUCTURE ONLY: the
checker for snc_b200.bptt and the "autograd bridge" leg of the benchmarks.

Follows python/snc/model.py:
  * SurrogateSpike (:17-30): Heaviside forward, fast-sigmoid backward
    g / (1 + k|x|)^2 -- here k is an argument instead of the class attribute
    the reference mutates globally;
  * SNN.forward (:52-72): msg = w * s[:, pre]; cur = index_add over post;
    v = decay * v + cur + ext; s = H(v - thr); v = v * (1 - s);
and the delayed recurrence of python/snc/shd_model.py:109-121,143-145
(spike history s_hist[delay - 1, :, pre]).  A spike at step t reaches its
post at step t + delay (the reference's delay-1 model is the special case).

``smooth=True`` replaces the Heaviside by s = x / (1 + k|x|), whose exact
derivative is the surrogate; finite differences of that model check the
backward formulas.
"""
from __future__ import annotations

import torch


class SurrogateSpike(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, k):
        ctx.save_for_backward(x)
        ctx.k = k
        return (x >= 0).to(x.dtype)

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        return g / (1.0 + ctx.k * x.abs()) ** 2, None


def spike_fn(x, k, smooth):
    if smooth:
        return x / (1.0 + k * x.abs())
    return SurrogateSpike.apply(x, k)


def core_forward(w, ext, pre, post, delays, thr, decay, k, smooth=False):
    """w [S], ext [T, B, N] -> spikes [T, B, N]; pre/post/delays [S] long."""
    T, B, N = ext.shape
    D = int(delays.max().item()) if delays.numel() else 1
    hist = torch.zeros(D, B, N, dtype=ext.dtype, device=ext.device)
    v = torch.zeros(B, N, dtype=ext.dtype, device=ext.device)
    out = []
    for t in range(T):
        src = hist[delays - 1, :, pre]                               # [S, B]
        cur = torch.zeros(B, N, dtype=ext.dtype, device=ext.device).index_add(
            1, post, (w.unsqueeze(1) * src).t())
        v = decay * v + cur + ext[t]
        s = spike_fn(v - thr, k, smooth)
        v = v * (1.0 - s)
        out.append(s)
        hist = torch.cat([s.unsqueeze(0), hist[:-1]], dim=0)
    return torch.stack(out)


def leaky_readout(spikes, w_ro, b_ro, ro_ids, ro_decay):
    """SHDNet's leaky readout (shd_model.py:139-140,147): out = ro_decay * out
    + Linear(s_top); logits = out / T after the last step."""
    T = spikes.shape[0]
    out = torch.zeros(spikes.shape[1], w_ro.shape[0], dtype=spikes.dtype, device=spikes.device)
    for t in range(T):
        out = ro_decay * out + torch.nn.functional.linear(spikes[t][:, ro_ids], w_ro, b_ro)
    return out / T
