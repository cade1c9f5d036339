"""Surrogate-gradient BPTT on the B200: the bridge's spiking core
(python/snc/model.py, python/snc/shd_model.py) with a hand-written forward
and backward over the sparse delayed graph, behind torch.autograd.Function.

  SpikingCore      device graph (CSR + incoming lists) of one spiking layer
  SNNFunction      autograd.Function: (w, ext) -> spikes; backward gives
                   dL/dw and dL/dext from dL/dspikes (include/snc_b200.h,
                   snc_b200_bptt_*)
  SNN              drop-in for python/snc/model.py SNN (same constructor and
                   forward), with per-synapse delays allowed
  DelayedSNN       784 -> hidden spiking graph with delays + leaky readout
  SpikingLM        embedding -> recurrent delayed spiking core -> leaky trace
                   -> linear readout (python/snc/lm.py, one layer)

PyTorch supplies device memory, the stream and the dense parts (input
encoding, embedding, readout); the spiking core runs in libsnc_b200.so.
"""
from __future__ import annotations

import ctypes as C
import sys

import numpy as np
import torch
import torch.nn as nn
import torch.nn.functional as F

from . import _lib
from ._lib import check, lib


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class SpikingCore:
    """One spiking graph on the device.  Edges are given as (pre, post,
    delay) in any order; they are kept in CSR order (stable by pre) and
    ``perm`` maps CSR positions back to the caller's order."""

    def __init__(self, num_neurons, pre, post, delays, device=None):
        pre = np.asarray(pre, np.int64)
        post = np.asarray(post, np.int64)
        delays = np.asarray(delays, np.int64)
        if delays.size and delays.min() < 1:
            raise ValueError("delays must be >= 1")
        self.N = int(num_neurons)
        self.S = int(pre.shape[0])
        self.perm = np.argsort(pre, kind="stable")
        self.identity = bool(np.array_equal(self.perm, np.arange(self.S)))
        row_ptr = np.zeros(self.N + 1, np.int32)
        np.cumsum(np.bincount(pre, minlength=self.N), out=row_ptr[1:])
        self.row_ptr = row_ptr
        self.post = np.ascontiguousarray(post[self.perm], np.int32)
        self.delays = np.ascontiguousarray(delays[self.perm], np.int32)
        self.max_delay = int(delays.max()) if self.S else 1
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        check(lib().snc_b200_set_device(dev.index or 0), "set_device")
        h = C.c_void_p()
        check(lib().snc_b200_bptt_create(self.N, self.S, self.row_ptr.ctypes.data,
                                         self.post.ctypes.data, self.delays.ctypes.data,
                                         C.byref(h)), "bptt_create")
        self.h = h
        self.perm_t = torch.as_tensor(self.perm, device=dev)

    def set_resident(self, enable: bool) -> None:
        """Allow (default) or forbid the resident launches that stage every
        neuron's edges in shared memory; results are identical either way."""
        check(lib().snc_b200_bptt_set_resident(self.h, int(bool(enable))), "bptt_set_resident")

    def to_csr(self, w):
        return w if self.identity else w[self.perm_t]

    def from_csr(self, w_csr):
        if self.identity:
            return w_csr
        out = torch.empty_like(w_csr)
        out[self.perm_t] = w_csr
        return out

    def release(self):
        if getattr(self, "h", None):
            lib().snc_b200_bptt_release(self.h)
            self.h = None

    def __del__(self, _finalizing=sys.is_finalizing):
        # a default argument outlives the module globals cleared at exit
        if not _finalizing():  # the library may already be unloaded
            self.release()


def _transpose(x, I, J, st_t, st_j, T):
    out = torch.empty(T, I, J, device=x.device, dtype=torch.float32)
    check(lib().snc_b200_transpose(_ptr(x), _ptr(out), T, I, J, st_t, st_j, _stream()), "transpose")
    return out


def _to_tnb(x):
    """[T, B, N] fp32 (a view with unit stride along N is read in place) ->
    contiguous [T, N, B], the kernels' batch-innermost layout."""
    T, B, N = x.shape
    x = x.float()
    if x.stride(2) != 1 or T > 65535:
        return x.permute(0, 2, 1).contiguous()
    return _transpose(x, N, B, x.stride(0), x.stride(1), T)


def _from_tnb(y):
    """Contiguous [T, N, B] -> contiguous [T, B, N]."""
    T, N, B = y.shape
    if T > 65535:
        return y.permute(0, 2, 1).contiguous()
    return _transpose(y, B, N, N * B, B, T)


class SNNFunction(torch.autograd.Function):
    """spikes [T, B, N] = core(w [S], ext [T, B, N]); fp32 CUDA tensors."""

    @staticmethod
    def forward(ctx, w, ext, core, threshold, decay, slope, ckpt_every, smooth):
        T, B, N = ext.shape
        if N != core.N:
            raise ValueError("ext has the wrong number of neurons")
        check(lib().snc_b200_set_device(ext.device.index or 0), "set_device")
        ext_t = _to_tnb(ext.detach())
        w_csr = core.to_csr(w.detach()).contiguous()
        KB = (B + 31) // 32
        dev = ext.device
        spikes = torch.empty(T, N, B, device=dev, dtype=torch.float32)
        bits = torch.empty(T, N, KB, device=dev, dtype=torch.int32)
        K = int(ckpt_every)
        vsaved = torch.empty((T + K - 1) // K if K > 0 else T, N, B, device=dev, dtype=torch.float32)
        check(lib().snc_b200_bptt_forward(core.h, _ptr(w_csr), _ptr(ext_t), T, B, float(threshold),
                                          float(decay), float(slope), K, int(bool(smooth)),
                                          _ptr(spikes), _ptr(bits), _ptr(vsaved), _stream()),
              "bptt_forward")
        ctx.core, ctx.args = core, (T, B, float(threshold), float(decay), float(slope), K, int(bool(smooth)))
        ctx.save_for_backward(w_csr, ext_t, spikes, bits, vsaved)
        return _from_tnb(spikes)

    @staticmethod
    def backward(ctx, g_spikes):
        w_csr, ext_t, spikes, bits, vsaved = ctx.saved_tensors
        core = ctx.core
        T, B, thr, decay, slope, K, smooth = ctx.args
        check(lib().snc_b200_set_device(ext_t.device.index or 0), "set_device")
        g_t = _to_tnb(g_spikes)
        grad_w = torch.empty(core.S, device=ext_t.device, dtype=torch.float32)
        want_ext = ctx.needs_input_grad[1]
        grad_ext = torch.empty_like(ext_t) if want_ext else None
        check(lib().snc_b200_bptt_backward(core.h, _ptr(w_csr), _ptr(ext_t), T, B, thr, decay, slope,
                                           K, smooth, _ptr(spikes), _ptr(bits), _ptr(vsaved),
                                           _ptr(g_t), _ptr(grad_w), _ptr(grad_ext), _stream()),
              "bptt_backward")
        gw = core.from_csr(grad_w) if ctx.needs_input_grad[0] else None
        ge = _from_tnb(grad_ext) if want_ext else None
        return gw, ge, None, None, None, None, None, None


def spiking_core(w, ext, core, threshold=1.0, decay=0.9, slope=10.0, ckpt_every=10, smooth=False):
    return SNNFunction.apply(w, ext, core, threshold, decay, slope, ckpt_every, smooth)


class SNN(nn.Module):
    """python/snc/model.py SNN with the same constructor and forward: x
    [B, dim] in [0,1] -> logits [B, n_out] (summed output spikes).  Poisson
    or direct drive into input neurons 0..dim-1.  Delays > 1 are allowed."""

    def __init__(self, g, num_steps=20, thr=1.0, decay=0.9, gain=1.0, max_rate=0.5, w_init=0.1,
                 surrogate_scale=10.0, encoder="poisson", seed=0, ckpt_every=10):
        super().__init__()
        self.N, self.dim, self.n_out = g["N"], g["n_in"], g["n_out"]
        self.T, self.thr, self.decay = num_steps, thr, decay
        self.gain, self.max_rate, self.encoder = gain, max_rate, encoder
        self.slope, self.ckpt_every = surrogate_scale, ckpt_every
        out_ids = np.where(np.asarray(g["role"]) == 2)[0]
        self.register_buffer("out_ids", torch.as_tensor(out_ids, dtype=torch.long))
        self.register_buffer("out_ch", torch.as_tensor(np.asarray(g["channel"])[out_ids], dtype=torch.long))
        self._edges = (np.asarray(g["pre"]), np.asarray(g["post"]), np.asarray(g["delays"]))
        self._core = None
        gen = torch.Generator().manual_seed(seed)
        self.w = nn.Parameter((torch.rand(g["S"], generator=gen) * 2 - 1) * w_init)

    def core(self):
        if self._core is None or self._core.device != self.w.device:
            self._core = SpikingCore(self.N, *self._edges, device=self.w.device)
        return self._core

    def forward(self, x):
        B, dev = x.shape[0], self.w.device
        if self.encoder == "poisson":
            inp = (torch.rand(self.T, B, self.dim, device=dev) < x * self.max_rate).float()
        else:
            inp = x.unsqueeze(0).expand(self.T, B, self.dim)
        ext = torch.zeros(self.T, B, self.N, device=dev)
        ext[:, :, :self.dim] = inp * self.gain
        s = spiking_core(self.w, ext, self.core(), self.thr, self.decay, self.slope, self.ckpt_every)
        return torch.zeros(B, self.n_out, device=dev).index_add(1, self.out_ch, s.sum(0)[:, self.out_ids])


class LeakyScan(torch.autograd.Function):
    """y[t] = decay * y[t-1] + x[t] along dim 0 of a [T, ...] fp32 CUDA tensor
    (snc_b200_leaky_scan): the leaky readout loops of shd_model.py:139-140 and
    lm.py:90 in one kernel, same roundings; the gradient is the reverse scan."""

    @staticmethod
    def forward(ctx, x, decay):
        x = x.contiguous().float()
        y = torch.empty_like(x)
        T = x.shape[0]
        check(lib().snc_b200_leaky_scan(_ptr(x), _ptr(y), T, x.numel() // max(1, T), float(decay), 0,
                                        _stream()), "leaky_scan")
        ctx.decay = float(decay)
        return y

    @staticmethod
    def backward(ctx, g):
        g = g.contiguous().float()
        gx = torch.empty_like(g)
        T = g.shape[0]
        check(lib().snc_b200_leaky_scan(_ptr(g), _ptr(gx), T, g.numel() // max(1, T), ctx.decay, 1,
                                        _stream()), "leaky_scan")
        return gx, None


def leaky_scan(x, decay):
    return LeakyScan.apply(x, decay)


class DelayedSNN(nn.Module):
    """Input spikes -> sparse delayed spiking graph -> leaky readout
    (shd_model.py leaky readout: out = ro_decay*out + Linear(s_top),
    logits = out / T).  ext is built from pre-generated input spikes
    [T, B, n_in] driving neurons 0..n_in-1."""

    def __init__(self, num_neurons, pre, post, delays, n_in, readout_ids, n_class, thr=1.0,
                 decay=0.95, gain=1.0, surrogate_scale=25.0, ro_decay=0.9, w_init=None, seed=0,
                 ckpt_every=10, device=None):
        super().__init__()
        self.N, self.n_in, self.thr, self.decay = num_neurons, n_in, thr, decay
        self.gain, self.slope, self.ro_decay, self.ckpt_every = gain, surrogate_scale, ro_decay, ckpt_every
        gen = torch.Generator().manual_seed(seed)
        S = len(pre)
        w = torch.as_tensor(w_init, dtype=torch.float32) if w_init is not None else \
            (torch.rand(S, generator=gen) * 2 - 1) * 0.5
        self.w = nn.Parameter(w)
        self.register_buffer("ro_ids", torch.as_tensor(readout_ids, dtype=torch.long))
        self.readout = nn.Linear(len(readout_ids), n_class)
        self._edges = (np.asarray(pre), np.asarray(post), np.asarray(delays))
        self._core = None

    def core(self):
        if self._core is None or self._core.device != self.w.device:
            self._core = SpikingCore(self.N, *self._edges, device=self.w.device)
        return self._core

    def forward(self, spikes_in):  # [T, B, n_in] -> logits [B, n_class]
        T, B, _ = spikes_in.shape
        ext = torch.zeros(T, B, self.N, device=self.w.device)
        ext[:, :, :self.n_in] = spikes_in * self.gain
        s = spiking_core(self.w, ext, self.core(), self.thr, self.decay, self.slope, self.ckpt_every)
        # out(T-1) of out = ro_decay * out + readout(s_top): the readout of the
        # leaky-integrated spikes plus the bias summed with the same decay
        r = leaky_scan(s.index_select(2, self.ro_ids), self.ro_decay)[T - 1]
        bias_gain = float(sum(self.ro_decay ** k for k in range(T)))
        out = F.linear(r, self.readout.weight) + self.readout.bias * bias_gain
        return out / T


class SpikingLM(nn.Module):
    """python/snc/lm.py SpikingLM with one recurrent layer and per-synapse
    delays: token -> Embed -> input current; r = ro_decay*r + s;
    logits(t) = Readout(r(t))."""

    def __init__(self, vocab, hidden, pre, post, delays, decay=0.95, thr=1.0, ro_decay=0.9,
                 surrogate_scale=25.0, w_scale=0.5, seed=0, ckpt_every=16):
        super().__init__()
        self.vocab, self.H = vocab, hidden
        self.decay, self.thr, self.ro_decay = decay, thr, ro_decay
        self.slope, self.ckpt_every = surrogate_scale, ckpt_every
        self.embed = nn.Embedding(vocab, hidden)
        self.readout = nn.Linear(hidden, vocab)
        gen = torch.Generator().manual_seed(seed)
        post_t = torch.as_tensor(np.asarray(post), dtype=torch.long)
        fanin = torch.zeros(hidden).index_add(0, post_t, torch.ones(post_t.numel())).clamp_min_(1.0)
        w = (torch.rand(len(pre), generator=gen) * 2 - 1) * w_scale
        self.w_rec = nn.Parameter(w / fanin[post_t].sqrt())
        self._edges = (np.asarray(pre), np.asarray(post), np.asarray(delays))
        self._core = None

    def core(self):
        if self._core is None or self._core.device != self.w_rec.device:
            self._core = SpikingCore(self.H, *self._edges, device=self.w_rec.device)
        return self._core

    def forward(self, x):  # [B, T] token ids -> logits [B, T, vocab]
        B, T = x.shape
        ext = self.embed(x).transpose(0, 1)                       # [T, B, H]
        s = spiking_core(self.w_rec, ext, self.core(), self.thr, self.decay, self.slope,
                         self.ckpt_every)
        r = leaky_scan(s, self.ro_decay)                          # [T, B, H]
        return self.readout(r.transpose(0, 1))
