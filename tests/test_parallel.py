"""Sample-sharded data-parallel e-prop on CPU ranks (gloo, world size 2).

The GPU session is replaced by a stand-in that computes each shard's
gradient with the CPU restatement and applies the update with the same
operation order as snc_b200_eprop_apply; the test checks the sharding, the
all-reduce and the update rule: every rank ends with identical weights, equal
(up to float summation order) to one minibatch over all samples."""
import os

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O
from snc_b200 import parallel as PAR
from snc_b200 import runtime as R
from snc_b200 import workloads as W
from snc_b200.graph import INTERNAL

LR, WMAX, GAMMA, TD = 0.7, 4.0, 0.3, 0.95


def case():
    g = W.random_graph(11, n_hid=50, max_delay=5)
    ev, st = W.random_events(12, g, 5, [30, 18, 30, 25, 9])
    rng = np.random.default_rng(3)
    w0 = rng.normal(0, 0.5, g.num_synapses).astype(np.float32)
    fb = rng.normal(0, 1.0, (int((g.role == INTERNAL).sum()), g.num_output_channels)).astype(np.float32)
    labels = rng.integers(0, g.num_output_channels, 5).astype(np.int32)
    return g, ev, st, w0, fb, labels


class OracleSession:
    def __init__(self, g, w, fb):
        self.g, self.w, self.fb = g, w.copy(), fb
        self.lif = R.LIFParams(refractory=1)

    def gradient(self, ev, st, lab, grad):
        r = O.eprop_batch(self.g, self.w, ev, st, self.lif, trace_decay=TD, gamma=GAMMA, lr=LR,
                          w_max=WMAX, train_hidden=True, bmat=self.fb, labels=lab, want_grad=True)
        grad.copy_(torch.from_numpy(r["grad"]))
        return r

    def apply(self, grad, total_batch):
        gv = grad.numpy().astype(np.float32)
        nw = self.w - (np.float32(LR) * gv) / np.float32(total_batch)
        self.w = np.clip(nw, -WMAX, WMAX).astype(np.float32)


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, ev, st, w0, fb, labels = case()
        s = OracleSession(g, w0, fb)
        PAR.DataParallelEprop(s, g.num_synapses, device="cpu").step(ev, st, labels)
        np.save(os.path.join(out, f"w{rank}.npy"), s.w)
    finally:
        dist.destroy_process_group()


def test_shard_bounds_cover_all_samples():
    for n in (0, 1, 5, 7, 64):
        for world in (1, 2, 3, 8):
            spans = [PAR.shard_bounds(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
            assert max(h - l for l, h in spans) - min(h - l for l, h in spans) <= 1


def test_shard_samples_renumbers():
    g, ev, st, w0, fb, labels = case()
    ev1, st1, lab1 = PAR.shard_samples(ev, st, labels, 1, 2)
    assert list(st1) == [25, 9] and list(lab1) == list(labels[3:5])
    assert set(np.unique(ev1["sample_id"])) <= {0, 1}
    assert len(ev1) == int(((ev["sample_id"] >= 3) & (ev["sample_id"] < 5)).sum())


def test_data_parallel_eprop_gloo_world2(tmp_path):
    port = 29500 + (os.getpid() % 1000)
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    w_r0 = np.load(tmp_path / "w0.npy")
    w_r1 = np.load(tmp_path / "w1.npy")
    np.testing.assert_array_equal(w_r0, w_r1)
    g, ev, st, w0, fb, labels = case()
    single = O.eprop_batch(g, w0, ev, st, R.LIFParams(refractory=1), trace_decay=TD, gamma=GAMMA,
                           lr=LR, w_max=WMAX, train_hidden=True, bmat=fb, labels=labels)
    assert np.abs(single["w"] - w0).max() > 0
    np.testing.assert_allclose(w_r0, single["w"], rtol=1e-5, atol=1e-6)


# ---- post-neuron partitioned forward (restatement on gloo ranks) ---------------

def part_case():
    g = W.rec100k_graph(seed=4, n=3000, width=60, out_degree=30, long_range=3, max_delay=12)
    ev, st = W.rec100k_inputs(g, 1, 120, rate=0.08, seed=2)
    return g, ev, int(st[0]), W.lif_tau20()


def _part_worker(rank, world, port, out):
    from oracle import partition as OP
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, ev, T, lif = part_case()
        N = g.num_neurons
        bounds = [(r * N // world, (r + 1) * N // world) for r in range(world)]
        lo, hi = bounds[rank]
        width = max(h - l for l, h in bounds)

        def gather(bits):
            buf = torch.zeros(width, dtype=torch.uint8)
            buf[:bits.shape[0]] = torch.from_numpy(bits.astype(np.uint8))
            parts = [torch.zeros(width, dtype=torch.uint8) for _ in range(world)]
            dist.all_gather(parts, buf)
            return np.concatenate([p.numpy()[:h - l] for p, (l, h) in zip(parts, bounds)]).astype(bool)

        r = OP.partition_forward(g, ev, T, lif, lo, hi, gather)
        np.savez(os.path.join(out, f"part{rank}.npz"), raster=r["raster"], v=r["v"],
                 counts=np.array([r["spikes"], r["events"]]), logits=r["logits"], lo=lo, hi=hi)
    finally:
        dist.destroy_process_group()


def test_partitioned_forward_gloo_world2_equals_single_rank(tmp_path):
    """Two gloo ranks, each owning half of the neurons, exchange one step's
    spike bits per step; together they reproduce the single-process forward
    bit for bit (rasters, potentials, spike and event counts, logits)."""
    port = 29700 + (os.getpid() % 1000)
    mp.start_processes(_part_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    g, ev, T, lif = part_case()
    ref = O.forward_batched(g, ev, np.array([T], np.int32), lif)
    parts = [np.load(tmp_path / f"part{r}.npz") for r in range(2)]
    raster = parts[0]["raster"] | parts[1]["raster"]
    np.testing.assert_array_equal(raster, ref["raster"])
    v = np.concatenate([p["v"] for p in parts])
    np.testing.assert_array_equal(v.view(np.uint32), ref["v"][0].view(np.uint32))
    assert sum(int(p["counts"][0]) for p in parts) == int(ref["spikes"][0]) > 0
    assert sum(int(p["counts"][1]) for p in parts) == int(ref["events"][0])
    np.testing.assert_array_equal(parts[0]["logits"] + parts[1]["logits"], ref["logits"][0])


def test_part_block_bounds_cover_the_blocks():
    for P in (1, 7, 125, 143):
        for world in (1, 2, 3, 8):
            if world > P:
                continue
            spans = [PAR.part_block_bounds(P, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == P
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))


# ---- sample-sharded BPTT (DataParallelBPTT on gloo ranks) ----------------------

class _RefDelayedSNN(torch.nn.Module):
    """CPU stand-in for snc_b200.bptt.DelayedSNN: the autograd restatement
    of the delayed spiking core and its leaky readout (the kernels need a
    GPU; the sharding, all-reduce and update logic under test do not)."""

    def __init__(self, g, n_in, ro_ids, n_class):
        super().__init__()
        from oracle import bptt_ref as BR
        self.BR = BR
        gen = torch.Generator().manual_seed(5)
        self.w = torch.nn.Parameter((torch.rand(g.num_synapses, generator=gen) * 2 - 1) * 0.6)
        self.readout = torch.nn.Linear(len(ro_ids), n_class)
        with torch.no_grad():
            self.readout.weight.copy_(torch.randn(self.readout.weight.shape, generator=gen) * 0.3)
            self.readout.bias.copy_(torch.randn(n_class, generator=gen) * 0.1)
        self.N, self.n_in = g.num_neurons, n_in
        self.pre = torch.as_tensor(g.pre_ids()).long()
        self.post = torch.as_tensor(g.post_ids).long()
        self.delays = torch.as_tensor(g.delays).long()
        self.ro_ids = torch.as_tensor(ro_ids).long()

    def forward(self, spikes_in):
        T, B, _ = spikes_in.shape
        ext = torch.zeros(T, B, self.N)
        ext[:, :, :self.n_in] = spikes_in
        s = self.BR.core_forward(self.w, ext, self.pre, self.post, self.delays, 1.0, 0.9, 25.0)
        return self.BR.leaky_readout(s, self.readout.weight, self.readout.bias, self.ro_ids, 0.9)


def bptt_case():
    g = W.random_graph(8, n_in=12, n_hid=30, n_out=4, max_delay=3)
    ro_ids = np.nonzero(np.asarray(g.role) == 2)[0]
    T, B = 16, 5
    x = (torch.rand(T, B, 12, generator=torch.Generator().manual_seed(3)) < 0.35).float()
    y = torch.as_tensor(np.random.default_rng(2).integers(0, 3, B))
    return g, ro_ids, x, y


def _bptt_loss(m, xs, ys):
    return torch.nn.functional.cross_entropy(m(xs), ys, reduction="sum")


def _bptt_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g, ro_ids, x, y = bptt_case()
        torch.manual_seed(0)
        m = _RefDelayedSNN(g, 12, ro_ids, 3)
        opt = torch.optim.SGD(m.parameters(), lr=0.5)
        loss = PAR.DataParallelBPTT(m, opt, _bptt_loss, batch_dim=1).step(x, y)
        torch.save({"w": m.w.detach(), "rw": m.readout.weight.detach(),
                    "rb": m.readout.bias.detach(), "loss": loss}, os.path.join(out, f"b{rank}.pt"))
    finally:
        dist.destroy_process_group()


def test_data_parallel_bptt_gloo_world2(tmp_path):
    """Two gloo ranks take one SGD step on uneven shards (3 + 2 samples) of a
    5-sample minibatch: both end with identical parameters, equal (up to
    float summation order) to one step on the whole batch's mean loss."""
    port = 29900 + (os.getpid() % 1000)
    mp.start_processes(_bptt_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r0 = torch.load(tmp_path / "b0.pt")
    r1 = torch.load(tmp_path / "b1.pt")
    for k in ("w", "rw", "rb"):
        assert torch.equal(r0[k], r1[k])
    g, ro_ids, x, y = bptt_case()
    torch.manual_seed(0)
    m = _RefDelayedSNN(g, 12, ro_ids, 3)
    w0 = m.w.detach().clone()
    opt = torch.optim.SGD(m.parameters(), lr=0.5)
    loss = torch.nn.functional.cross_entropy(m(x), y)
    loss.backward()
    opt.step()
    assert float((m.w.detach() - w0).abs().max()) > 0
    torch.testing.assert_close(r0["w"], m.w.detach(), rtol=1e-5, atol=1e-6)
    torch.testing.assert_close(r0["rw"], m.readout.weight.detach(), rtol=1e-5, atol=1e-6)
    torch.testing.assert_close(r0["rb"], m.readout.bias.detach(), rtol=1e-5, atol=1e-6)
    assert abs(r0["loss"] - float(loss)) <= 1e-5 * abs(float(loss))
