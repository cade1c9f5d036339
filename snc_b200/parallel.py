"""Sample-sharded data parallelism, one process per GPU.

Samples are independent under a frozen graph (include/snc/cuda_trainer.hpp:
5-7), so a minibatch splits into contiguous blocks of samples, one per rank:
  * forward / evaluation: no exchange (bench.py runs replicas);
  * e-prop: each rank computes the gradient of its shard
    (snc_b200_eprop_gradient), one all-reduce (sum) adds the shards, every
    rank applies the same update with the global batch size
    (snc_b200_eprop_apply) -- the weights stay identical on all ranks;
  * BPTT: SNNFunction returns ordinary autograd gradients; DataParallelBPTT
    computes each rank's shard gradient of the summed loss, adds the shards
    with one all-reduce of a single flat buffer and divides by the global
    batch, so uneven shards give the gradient of the global mean loss (DDP's
    averaging over ranks assumes equal shards).
The collective is torch.distributed (NCCL over NVLink on GPUs, gloo in the
CPU tests).  Remote data always arrives in local memory through NCCL; no
kernel here reads a peer's memory.
"""
from __future__ import annotations

import numpy as np


def shard_bounds(n: int, rank: int, world: int):
    """Contiguous [lo, hi) block of n samples for `rank` of `world` (the
    first n % world ranks take one extra sample)."""
    base, rem = divmod(n, world)
    lo = rank * base + min(rank, rem)
    return lo, lo + base + (1 if rank < rem else 0)


def shard_samples(events, steps, labels, rank: int, world: int):
    """The events, step counts and labels of this rank's samples, with
    sample ids renumbered from 0."""
    steps = np.asarray(steps)
    lo, hi = shard_bounds(steps.shape[0], rank, world)
    if events is not None and len(events):
        sel = (events["sample_id"] >= lo) & (events["sample_id"] < hi)
        ev = events[sel].copy()
        ev["sample_id"] -= lo
    else:
        ev = events
    lab = None if labels is None else np.asarray(labels)[lo:hi]
    return ev, steps[lo:hi], lab


class DataParallelEprop:
    """One e-prop update over a global minibatch split across ranks.

    ``session`` provides ``gradient(events, steps, labels, grad)`` and
    ``apply(grad, total_batch)`` (snc_b200.eprop.CudaTrainSession does);
    ``num_synapses`` sizes the gradient buffer on ``device``."""

    def __init__(self, session, num_synapses: int, device="cuda", group=None):
        self.session = session
        self.S = int(num_synapses)
        self.device = device
        self.group = group

    def step(self, events, steps, labels):
        import torch
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            world, rank = dist.get_world_size(self.group), dist.get_rank(self.group)
        else:
            world, rank = 1, 0
        ev, st, lab = shard_samples(events, steps, labels, rank, world)
        grad = torch.zeros(self.S, dtype=torch.float32, device=self.device)
        out = None
        if st.shape[0]:
            out = self.session.gradient(ev, st, lab, grad)
        if world > 1:
            dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=self.group)
        self.session.apply(grad, int(np.asarray(steps).shape[0]))
        return out


def shard_gradient(model, loss_fn, inputs, targets, batch_dim: int, rank: int, world: int):
    """This rank's share of one BPTT minibatch: the gradient of the SUMMED
    loss over its contiguous block of samples (shard_bounds), flattened over
    model.parameters() in order (zeros for a parameter without a gradient or
    an empty shard), and the summed loss.  loss_fn(model, x, y) returns the
    sum of per-sample losses of its samples."""
    import torch
    B = inputs.shape[batch_dim]
    lo, hi = shard_bounds(B, rank, world)
    params = [p for p in model.parameters()]
    for p in params:
        p.grad = None
    loss = torch.zeros((), dtype=torch.float64, device=params[0].device)
    if hi > lo:
        x = inputs.narrow(batch_dim, lo, hi - lo)
        y = targets[lo:hi]
        ls = loss_fn(model, x, y)
        ls.backward()
        loss = ls.detach().to(torch.float64)
    flat = torch.cat([(p.grad if p.grad is not None else torch.zeros_like(p)).reshape(-1).float()
                      for p in params])
    return flat, loss


class DataParallelBPTT:
    """One BPTT update over a global minibatch split across ranks: every rank
    computes its shard's gradient of the summed loss (shard_gradient), one
    all-reduce (sum) of the flat gradient and the loss adds the shards, the
    sum is divided by the global batch and written back to the parameters'
    .grad, and every rank takes the same optimizer step -- parameters stay
    identical on all ranks.  batch_dim is the inputs' sample dimension (1 for
    the [T, B, ...] spike tensors of DelayedSNN, 0 for SpikingLM's [B, T]
    tokens); targets are indexed by sample along dimension 0."""

    def __init__(self, model, optimizer, loss_fn, batch_dim: int, group=None):
        self.model, self.optimizer, self.loss_fn = model, optimizer, loss_fn
        self.batch_dim, self.group = batch_dim, group

    def step(self, inputs, targets):
        import torch
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            world, rank = dist.get_world_size(self.group), dist.get_rank(self.group)
        else:
            world, rank = 1, 0
        B = inputs.shape[self.batch_dim]
        flat, loss = shard_gradient(self.model, self.loss_fn, inputs, targets, self.batch_dim, rank,
                                    world)
        buf = torch.cat([flat, loss.float().reshape(1)])
        if world > 1:
            dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=self.group)
        buf /= float(B)
        off = 0
        for p in self.model.parameters():
            n = p.numel()
            p.grad = buf[off:off + n].view_as(p).to(p.dtype).clone()
            off += n
        self.optimizer.step()
        return float(buf[-1])


def part_block_bounds(num_blocks: int, rank: int, world: int):
    """Neuron blocks [lo, hi) of `rank` in a post-neuron partition: ceil(P /
    world) blocks per rank, so rank r's spike-bit words start at r times one
    rank's word count and an all-gather of equal chunks lands every word in
    its place."""
    per = -(-num_blocks // world)
    lo = min(num_blocks, rank * per)
    return lo, min(num_blocks, lo + per)


class PartitionedForward:
    """One sample's forward split by post neuron across ranks
    (snc_b200_part_*): each rank owns a contiguous range of neuron blocks --
    their state and ring columns -- and keeps the whole graph; per step the
    ranks integrate their neurons, all-gather the step's spike bits (ceil(N /
    32) words, 12.5 KB for 100k neurons: NCCL over NVLink on GPUs, landing in
    local memory), and deliver every fired neuron's synapses into their own
    columns in the CPU backend's order.  The ranks' results together equal a
    single-device SORT run bit for bit.  world == 1 needs no process group."""

    def __init__(self, dg, inputs, lif, rank=0, world=1, group=None):
        import ctypes as C
        import torch
        from ._lib import check, lib
        self.dg, self.inputs, self.rank, self.world, self.group = dg, inputs, rank, world, group
        self.T = int(inputs.steps[0])
        BS, P = dg.blocks()
        self.BS, self.P = BS, P
        self.blk = part_block_bounds(P, rank, world)
        if self.blk[0] >= self.blk[1]:
            raise ValueError("more ranks than neuron blocks")
        self.chunk = -(-P // world) * BS // 32
        self.words = (dg.N + 31) // 32
        self.mask = torch.zeros(world * self.chunk, dtype=torch.int32, device="cuda")
        lf = lif.c()
        h = C.c_void_p()
        check(lib().snc_b200_part_create(dg.h, inputs.h, self.blk[0], self.blk[1], C.byref(lf),
                                         C.byref(h)), "part_create")
        self.h = h

    def run(self):
        import ctypes as C
        import torch
        import torch.distributed as dist
        from ._lib import check, lib
        L = lib()
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        mp = C.c_void_p(self.mask.data_ptr())
        own = self.mask[self.rank * self.chunk:(self.rank + 1) * self.chunk]
        for t in range(self.T):
            check(L.snc_b200_part_integrate(self.h, t, mp, st), "part_integrate")
            if self.world > 1:
                dist.all_gather_into_tensor(self.mask, own.clone(), group=self.group)
            check(L.snc_b200_part_deliver(self.h, t, mp, st), "part_deliver")
        return self.fetch()

    def fetch(self):
        from ._lib import check, lib, ptr
        N, noc = self.dg.N, max(1, self.dg.n_out)
        logits = np.zeros(noc, np.float32)
        sp, ev = np.zeros(1, np.int64), np.zeros(1, np.int64)
        raster = np.zeros((self.T, self.words), np.uint32)
        v = np.zeros(N, np.float32)
        check(lib().snc_b200_part_fetch(self.h, ptr(logits), ptr(sp), ptr(ev), ptr(raster), ptr(v)),
              "part_fetch")
        lo, hi = self.blk[0] * self.BS, min(N, self.blk[1] * self.BS)
        return {"logits": logits[:self.dg.n_out], "spikes": int(sp[0]), "events": int(ev[0]),
                "raster": raster, "v": v[lo:hi], "neurons": (lo, hi)}

    def release(self):
        if getattr(self, "h", None):
            from ._lib import lib
            lib().snc_b200_part_release(self.h)
            self.h = None


def run_partitions_on_one_device(dg, inputs, lif, world):
    """`world` partitions of one sample stepped in turn on the current device
    with one shared spike-bit buffer (each step: every partition integrates,
    then every partition delivers): the partitioned mode's kernels without a
    process group.  Returns the per-partition results."""
    import ctypes as C
    import torch
    from ._lib import check, lib
    parts = [PartitionedForward.__new__(PartitionedForward) for _ in range(world)]
    BS, P = dg.blocks()
    chunk = -(-P // world) * BS // 32
    mask = torch.zeros(world * chunk, dtype=torch.int32, device="cuda")
    lf = lif.c()
    for r, p in enumerate(parts):
        p.dg, p.inputs, p.rank, p.world, p.group = dg, inputs, r, world, None
        p.T, p.BS, p.P = int(inputs.steps[0]), BS, P
        p.blk = part_block_bounds(P, r, world)
        if p.blk[0] >= p.blk[1]:
            raise ValueError("more partitions than neuron blocks")
        p.chunk, p.words, p.mask = chunk, (dg.N + 31) // 32, mask
        h = C.c_void_p()
        check(lib().snc_b200_part_create(dg.h, inputs.h, p.blk[0], p.blk[1], C.byref(lf), C.byref(h)),
              "part_create")
        p.h = h
    L = lib()
    st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    mp = C.c_void_p(mask.data_ptr())
    for t in range(parts[0].T):
        for p in parts:
            check(L.snc_b200_part_integrate(p.h, t, mp, st), "part_integrate")
        for p in parts:
            check(L.snc_b200_part_deliver(p.h, t, mp, st), "part_deliver")
    out = [p.fetch() for p in parts]
    for p in parts:
        p.release()
    return out
