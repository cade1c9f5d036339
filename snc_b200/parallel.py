"""Sample-sharded data parallelism, one process per GPU.

Samples are independent under a frozen graph (include/snc/cuda_trainer.hpp:
5-7), so a minibatch splits into contiguous blocks of samples, one per rank:
  * forward / evaluation: no exchange (bench.py runs replicas);
  * e-prop: each rank computes the gradient of its shard
    (snc_b200_eprop_gradient), one all-reduce (sum) adds the shards, every
    rank applies the same update with the global batch size
    (snc_b200_eprop_apply) -- the weights stay identical on all ranks;
  * BPTT: SNNFunction returns ordinary gradients, so the models work under
    torch.nn.parallel.DistributedDataParallel unchanged.
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
