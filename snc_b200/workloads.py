"""Seeded synthetic graphs and inputs for the benchmark configurations.

No dataset is read: every graph, weight, label and input spike train is drawn
from numpy's PCG64 generator with a fixed seed, with the shapes and value
distributions the configurations specify.

  ff784     784 Poisson inputs -> 256 LIF -> 10 LIF, fan-in 32 by 2-D locality
            (Gaussian, sigma 3 grid units), w ~ N(0, 0.1), delays U{1..4};
            50 steps x 64 samples, rate = uniform[0,1] intensity x 0.2.
  rec100k   100k LIF on a 400 x 250 torus, out-degree 100 (95 local by a
            Gaussian displacement weighted by a lognormal(0, 1) target
            attractiveness -> heavy-tailed in-degree, 5 uniform long-range),
            w ~ N(0, 0.05), delays U{1..30}; 10% of neurons get Poisson drive
            at 0.02 / step; 1000 steps, batch 1.
  audio700  256 samples, 700 input channels, T_b ~ U{50..1000}, per-channel
            rates lognormal(mean 0.01, sigma 1); 1024 LIF recurrent at 10%,
            input projection 10%, 20 output units, delays U{1..30}.

All LIF neurons use tau_mem = 20 (decay = exp(-1/20)), threshold 1.0,
subtractive reset and no refractory period.
"""
from __future__ import annotations

import math

import numpy as np

from .graph import EVENT_DTYPE, INPUT, INTERNAL, OUTPUT, SNNGraph

DECAY_TAU20 = float(np.float32(math.exp(-1.0 / 20.0)))


def lif_tau20():
    from .runtime import LIFParams
    return LIFParams(threshold=1.0, decay=DECAY_TAU20, reset=0.0, refractory=0, reset_mode=1)


def _grid(nx, ny, extent):
    xs, ys = np.meshgrid(np.arange(nx), np.arange(ny), indexing="xy")
    sx = extent / max(nx - 1, 1)
    sy = extent / max(ny - 1, 1)
    return np.stack([xs.ravel() * sx, ys.ravel() * sy], axis=1)


def _local_fanin(rng, pre_pos, post_pos, k, sigma):
    """For each post, k distinct pres drawn without replacement with
    probability proportional to exp(-d^2 / (2 sigma^2)) (Gumbel top-k)."""
    d2 = ((post_pos[:, None, :] - pre_pos[None, :, :]) ** 2).sum(-1)
    keys = -d2 / (2 * sigma * sigma) + rng.gumbel(size=d2.shape)
    return np.argpartition(-keys, k - 1, axis=1)[:, :k]


def _csr_from_pairs(n, pre, post, w, d):
    order = np.lexsort((post, pre))
    pre, post, w, d = pre[order], post[order], w[order], d[order]
    row_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(pre, minlength=n), out=row_ptr[1:])
    return row_ptr.astype(np.int32), post.astype(np.int32), w.astype(np.float32), d.astype(np.int32)


def ff784_graph(seed=1, fan_in=32, sigma=3.0, w_std=0.1, max_delay=4) -> SNNGraph:
    rng = np.random.default_rng(seed)
    n_in, n_hid, n_out = 784, 256, 10
    N = n_in + n_hid + n_out
    p_in = _grid(28, 28, 27.0)
    p_hid = _grid(16, 16, 27.0)
    p_out = _grid(5, 2, 27.0)
    hid_pres = _local_fanin(rng, p_in, p_hid, fan_in, sigma)            # [256, 32] in [0,784)
    out_pres = _local_fanin(rng, p_hid, p_out, fan_in, sigma) + n_in    # [10, 32]
    pre = np.concatenate([hid_pres.ravel(), out_pres.ravel()])
    post = np.concatenate([np.repeat(np.arange(n_hid) + n_in, fan_in),
                           np.repeat(np.arange(n_out) + n_in + n_hid, fan_in)])
    S = pre.shape[0]
    w = rng.normal(0.0, w_std, S).astype(np.float32)
    d = rng.integers(1, max_delay + 1, S)
    role = np.full(N, INTERNAL, np.uint8)
    role[:n_in] = INPUT
    role[n_in + n_hid:] = OUTPUT
    channel = np.full(N, -1, np.int32)
    channel[:n_in] = np.arange(n_in)
    channel[n_in + n_hid:] = np.arange(n_out)
    rp, po, ww, dd = _csr_from_pairs(N, pre, post, w, d)
    return SNNGraph(N, rp, po, ww, dd, role, np.ones(N, np.int8), channel)


def poisson_events(rng, rates, num_steps, sample_id=0, amplitude=1.0) -> np.ndarray:
    """Bernoulli(rate_c) spike per (channel, step), channel-major then time
    (the order of snc::encode, encoders.cpp:43-55)."""
    rates = np.asarray(rates, dtype=np.float32)
    u = rng.random((rates.shape[0], num_steps), dtype=np.float32)
    c, t = np.nonzero(u < rates[:, None])
    ev = np.zeros(c.shape[0], dtype=EVENT_DTYPE)
    ev["sample_id"] = sample_id
    ev["channel_id"] = c
    ev["time"] = t
    ev["amplitude"] = amplitude
    return ev


def ff784_inputs(num_samples=64, num_steps=50, seed=1, max_rate=0.2):
    """Features ~ U[0,1] per (sample, channel); rate = feature x max_rate."""
    evs = []
    for i in range(num_samples):
        rng = np.random.default_rng([seed, i])
        x = rng.random(784, dtype=np.float32)
        evs.append(poisson_events(rng, x * np.float32(max_rate), num_steps, sample_id=i))
    return np.concatenate(evs), np.full(num_samples, num_steps, np.int32)


def rec100k_graph(seed=1, n=100_000, width=400, out_degree=100, long_range=5, sigma=4.0,
                  w_std=0.05, max_delay=30, input_frac=0.1, n_out=10, oversample=2) -> SNNGraph:
    rng = np.random.default_rng(seed)
    height = n // width
    assert width * height == n
    attract = rng.lognormal(0.0, 1.0, n).astype(np.float32)
    # accept a Gaussian-displaced candidate j with probability a_j / a_cap, so
    # local targets are drawn (with replacement) proportional to locality x a_j
    # and in-degree inherits the lognormal tail of a.
    acc = np.minimum(attract / np.float32(np.quantile(attract, 0.995)), 1.0)
    k_loc = out_degree - long_range
    posts = np.empty((n, out_degree), np.int32)
    m = int(k_loc * oversample * 2)
    got = np.zeros(n, np.int64)
    todo = np.arange(n)
    while todo.shape[0]:
        for c0 in range(0, todo.shape[0], 20000):
            ids = todo[c0:c0 + 20000]
            x, y = (ids % width).astype(np.int32), (ids // width).astype(np.int32)
            shape = (ids.shape[0], m)
            dx = np.rint(rng.standard_normal(shape, dtype=np.float32) * sigma).astype(np.int32)
            dy = np.rint(rng.standard_normal(shape, dtype=np.float32) * sigma).astype(np.int32)
            cand = ((y[:, None] + dy) % height) * width + (x[:, None] + dx) % width
            ok = rng.random(shape, dtype=np.float32) < acc[cand]
            g0 = got[ids]
            rank = np.cumsum(ok, axis=1) - 1 + g0[:, None]   # slot of each accepted candidate
            r, q = np.nonzero(ok & (rank < k_loc))
            posts[ids[r], rank[r, q]] = cand[r, q]
            got[ids] = np.minimum(g0 + ok.sum(axis=1), k_loc)
        todo = np.nonzero(got < k_loc)[0]
    posts[:, k_loc:] = rng.integers(0, n, (n, long_range))
    S = n * out_degree
    row_ptr = (np.arange(n + 1, dtype=np.int64) * out_degree).astype(np.int32)
    w = rng.normal(0.0, w_std, S).astype(np.float32)
    d = rng.integers(1, max_delay + 1, S).astype(np.int32)
    role = np.full(n, INTERNAL, np.uint8)
    channel = np.full(n, -1, np.int32)
    inp = np.sort(rng.choice(n, int(n * input_frac), replace=False))
    role[inp] = INPUT
    channel[inp] = np.arange(inp.shape[0])
    rest = np.setdiff1d(np.arange(n), inp)
    outs = np.sort(rng.choice(rest, n_out, replace=False))
    role[outs] = OUTPUT
    channel[outs] = np.arange(n_out)
    return SNNGraph(n, row_ptr, posts.ravel(), w, d, role, np.ones(n, np.int8), channel)


def rec100k_inputs(g: SNNGraph, num_samples=1, num_steps=1000, rate=0.02, seed=1):
    evs = []
    for i in range(num_samples):
        rng = np.random.default_rng([seed, 100 + i])
        evs.append(poisson_events(rng, np.full(g.num_input_channels, rate, np.float32), num_steps,
                                  sample_id=i))
    return np.concatenate(evs), np.full(num_samples, num_steps, np.int32)


def audio700_graph(seed=1, n_in=700, n_rec=1024, n_out=20, p=0.1, max_delay=30,
                   w_in=0.5, w_rec=0.1, w_out=0.1) -> SNNGraph:
    rng = np.random.default_rng(seed)
    N = n_in + n_rec + n_out
    rec0, out0 = n_in, n_in + n_rec
    pres, posts, ws = [], [], []
    a, b = np.nonzero(rng.random((n_in, n_rec)) < p)
    pres.append(a); posts.append(b + rec0); ws.append(rng.normal(0, w_in, a.shape[0]))
    a, b = np.nonzero(rng.random((n_rec, n_rec)) < p)
    keep = a != b
    a, b = a[keep], b[keep]
    pres.append(a + rec0); posts.append(b + rec0); ws.append(rng.normal(0, w_rec, a.shape[0]))
    a, b = np.nonzero(np.ones((n_rec, n_out), bool))
    pres.append(a + rec0); posts.append(b + out0); ws.append(rng.normal(0, w_out, a.shape[0]))
    pre, post, w = np.concatenate(pres), np.concatenate(posts), np.concatenate(ws)
    d = rng.integers(1, max_delay + 1, pre.shape[0])
    role = np.full(N, INTERNAL, np.uint8)
    role[:n_in] = INPUT
    role[out0:] = OUTPUT
    channel = np.full(N, -1, np.int32)
    channel[:n_in] = np.arange(n_in)
    channel[out0:] = np.arange(n_out)
    rp, po, ww, dd = _csr_from_pairs(N, pre, post, w, d)
    return SNNGraph(N, rp, po, ww, dd, role, np.ones(N, np.int8), channel)


def audio700_inputs(num_samples=256, t_min=50, t_max=1000, mean_rate=0.01, sigma=1.0, seed=1,
                    n_in=700):
    rng0 = np.random.default_rng([seed, 7])
    steps = rng0.integers(t_min, t_max + 1, num_samples).astype(np.int32)
    mu = math.log(mean_rate) - 0.5 * sigma * sigma
    evs = []
    for i in range(num_samples):
        rng = np.random.default_rng([seed, 1000 + i])
        rates = np.minimum(rng.lognormal(mu, sigma, n_in), 1.0).astype(np.float32)
        evs.append(poisson_events(rng, rates, int(steps[i]), sample_id=i))
    return np.concatenate(evs), steps


def random_graph(seed, n_in=20, n_hid=60, n_out=5, p=0.15, max_delay=5, recurrent=True,
                 inhib=0.2, w_scale=0.6, dup_frac=0.05) -> SNNGraph:
    """Small mixed test graph: feed-forward + recurrent edges, inhibitory
    neurons (negative sign), duplicate (pre, post) synapses with different
    delays, and neurons without incoming synapses."""
    rng = np.random.default_rng(seed)
    N = n_in + n_hid + n_out
    h0, o0 = n_in, n_in + n_hid
    pairs = []
    a, b = np.nonzero(rng.random((n_in, n_hid)) < p)
    pairs.append((a, b + h0))
    if recurrent:
        a, b = np.nonzero(rng.random((n_hid, n_hid)) < p)
        pairs.append((a + h0, b + h0))
    a, b = np.nonzero(rng.random((n_hid, n_out)) < 2 * p)
    pairs.append((a + h0, b + o0))
    pre = np.concatenate([x for x, _ in pairs])
    post = np.concatenate([y for _, y in pairs])
    ndup = int(dup_frac * pre.shape[0])
    if ndup:
        k = rng.integers(0, pre.shape[0], ndup)
        pre = np.concatenate([pre, pre[k]])
        post = np.concatenate([post, post[k]])
    perm = rng.permutation(pre.shape[0])
    pre, post = pre[perm], post[perm]
    w = np.abs(rng.normal(0, w_scale, pre.shape[0])).astype(np.float32)
    d = rng.integers(1, max_delay + 1, pre.shape[0]).astype(np.int32)
    order = np.argsort(pre, kind="stable")  # keep the shuffled order inside rows
    pre, post, w, d = pre[order], post[order], w[order], d[order]
    row_ptr = np.zeros(N + 1, np.int64)
    np.cumsum(np.bincount(pre, minlength=N), out=row_ptr[1:])
    role = np.full(N, INTERNAL, np.uint8)
    role[:n_in] = INPUT
    role[o0:] = OUTPUT
    channel = np.full(N, -1, np.int32)
    channel[:n_in] = np.arange(n_in) % max(1, n_in - 2)  # two channels drive two neurons
    channel[o0:] = np.arange(n_out)
    sign = np.where(rng.random(N) < inhib, -1, 1).astype(np.int8)
    sign[:n_in] = 1
    return SNNGraph(N, row_ptr.astype(np.int32), post, w, d, role, sign, channel)


def random_events(seed, g: SNNGraph, num_samples, steps, rate=0.2, amp_jitter=True):
    """Poisson input events for every sample, with duplicate events (the same
    channel twice in one step), out-of-range times and channels that the
    schedule must drop, and shuffled event order across samples."""
    rng = np.random.default_rng(seed)
    evs = []
    steps = np.broadcast_to(np.asarray(steps, np.int32), (num_samples,))
    for i in range(num_samples):
        ev = poisson_events(rng, np.full(g.num_input_channels, rate, np.float32), int(steps[i]),
                            sample_id=i)
        if amp_jitter:
            ev["amplitude"] = rng.uniform(0.5, 1.5, ev.shape[0]).astype(np.float32)
        extra = np.zeros(4, dtype=EVENT_DTYPE)
        extra["sample_id"] = i
        extra["channel_id"] = [0, g.num_input_channels + 3, 1, -1]
        extra["time"] = [0, 1, int(steps[i]) + 2, 0]
        extra["amplitude"] = [0.7, 5.0, 5.0, 5.0]
        evs.append(np.concatenate([ev, extra]))
    ev = np.concatenate(evs)
    return ev[rng.permutation(ev.shape[0])], np.array(steps, np.int32)


# ---------------------------------------------------------------------------
# BPTT workloads
# ---------------------------------------------------------------------------

def layered_local_edges(layers, fanout, seed=1, max_delay=4):
    """Feed-forward layers with 1-D local receptive fields: every pre in layer
    l projects to a contiguous window of `fanout` neurons of layer l+1 centred
    on its relative position (the make_static_snc pattern,
    src/graph/snn_graph.cpp:185-236).  Delays U{1..max_delay}."""
    rng = np.random.default_rng(seed)
    pres, posts = [], []
    base = 0
    for l in range(len(layers) - 1):
        a_n, b_n = layers[l], layers[l + 1]
        k = min(fanout, b_n)
        pos = np.arange(a_n) / max(1, a_n - 1)
        centre = np.clip(np.rint(pos * (b_n - 1)).astype(np.int64), 0, b_n - 1)
        lo = np.clip(centre - k // 2, 0, b_n - k)
        pres.append(np.repeat(np.arange(a_n) + base, k))
        posts.append((lo[:, None] + np.arange(k)[None, :]).ravel() + base + a_n)
        base += a_n
    pre, post = np.concatenate(pres), np.concatenate(posts)
    return pre, post, rng.integers(1, max_delay + 1, pre.shape[0])


def bptt_mnist_like(seed=1, T=100, B=128, rate=0.2):
    """784 Poisson inputs -> 512 -> 512 LIF (local sparse, ~6x fewer synapses
    than dense, delays 1-4) -> 10 leaky readout; input spikes [T, B, 784],
    random labels."""
    layers = [784, 512, 512]
    dense = 784 * 512 + 512 * 512
    fanout = int(round(dense / 6 / (784 + 512)))
    pre, post, d = layered_local_edges(layers, fanout, seed=seed, max_delay=4)
    rng = np.random.default_rng([seed, 2])
    x = rng.random((B, 784), dtype=np.float32) * np.float32(rate)
    spikes = (rng.random((T, B, 784), dtype=np.float32) < x[None]).astype(np.float32)
    labels = rng.integers(0, 10, B)
    readout_ids = np.arange(784 + 512, 784 + 1024)
    return {"N": 1808, "pre": pre, "post": post, "delays": d, "n_in": 784,
            "readout_ids": readout_ids, "spikes": spikes, "labels": labels}


def zipf_tokens(rng, vocab, n, s=1.1):
    p = 1.0 / np.arange(1, vocab + 1) ** s
    return rng.choice(vocab, size=n, p=p / p.sum())


def char_lm(seed=1, vocab=96, hidden=4096, fan_in=64, sigma=64.0, max_delay=8, B=64, T=256):
    """Spiking char-LM: recurrent hidden neurons with fan-in 64 drawn by a
    Gaussian over ring distance (locality-biased), delays U{1..8}; token ids
    from a seeded Zipf(1.1) sequence (no text corpus)."""
    rng = np.random.default_rng(seed)
    post = np.repeat(np.arange(hidden), fan_in)
    off = np.rint(rng.normal(0, sigma, post.shape[0])).astype(np.int64)
    off[off == 0] = 1
    pre = (post + off) % hidden
    order = np.argsort(pre, kind="stable")
    pre, post = pre[order], post[order]
    d = rng.integers(1, max_delay + 1, pre.shape[0])
    tokens = zipf_tokens(rng, vocab, B * (T + 1)).reshape(B, T + 1)
    return {"H": hidden, "vocab": vocab, "pre": pre, "post": post, "delays": d,
            "x": tokens[:, :T], "y": tokens[:, 1:]}


# ---- grid graphs from a counter-based generator ---------------------------------
# The rule snc_b200_graph_generate_grid runs on the device (csrc/generate.cu),
# restated with numpy so the same graph can be built on a host: Philox-4x32-10
# (Salmon et al., SC 2011) words counted by (neuron, draw, stream), integer
# arithmetic and single correctly rounded float32 operations only.

_PH_M0, _PH_M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_PH_W0, _PH_W1 = np.uint64(0x9E3779B9), np.uint64(0xBB67AE85)
_U32 = np.uint64(0xFFFFFFFF)


def _philox(c0, c1, c2, c3, seed):
    """Philox-4x32-10 of counters (c0, c1, c2, c3) (uint32 arrays) under key
    seed (64-bit); returns the four uint32 words."""
    c = [np.asarray(x, np.uint64) & _U32 for x in (c0, c1, c2, c3)]
    k0, k1 = np.uint64(seed & 0xFFFFFFFF), np.uint64((seed >> 32) & 0xFFFFFFFF)
    for _ in range(10):
        p0, p1 = _PH_M0 * c[0], _PH_M1 * c[2]
        c = [((p1 >> np.uint64(32)) ^ c[1] ^ k0) & _U32, p1 & _U32,
             ((p0 >> np.uint64(32)) ^ c[3] ^ k1) & _U32, p0 & _U32]
        k0, k1 = (k0 + _PH_W0) & _U32, (k1 + _PH_W1) & _U32
    return [x.astype(np.uint32) for x in c]


def _halves_sum(a, b):
    a, b = a.astype(np.int64), b.astype(np.int64)
    return (a >> 16) + (a & 0xFFFF) + (b >> 16) + (b & 0xFFFF) - 131072


def grid_graph_spec(seed=1, width=400, height=250, out_degree=100, long_range=5, sigma=4.0,
                    w_std=0.05, max_delay=30, input_frac=0.1, n_out=10, max_draws=0) -> dict:
    """Inputs of snc_b200_graph_generate_grid for a C2-style substrate (the
    defaults: 100k neurons, 10M synapses, delays 1-30): per-neuron acceptance
    thresholds from lognormal(0, 1) attractiveness capped at its 99.5 %
    quantile (the heavy-tailed in-degree), 10 % INPUT neurons and n_out
    OUTPUT neurons drawn with numpy from the seed."""
    n = width * height
    rng = np.random.default_rng([seed, 7])
    attract = rng.lognormal(0.0, 1.0, n)
    acc = np.minimum(attract / np.quantile(attract, 0.995), 1.0)
    accept = np.minimum(np.floor(acc * 4294967296.0), 4294967295.0).astype(np.uint32)
    role = np.full(n, INTERNAL, np.uint8)
    channel = np.full(n, -1, np.int32)
    inp = np.sort(rng.choice(n, int(n * input_frac), replace=False))
    role[inp] = INPUT
    channel[inp] = np.arange(inp.shape[0])
    rest = np.setdiff1d(np.arange(n), inp)
    outs = np.sort(rng.choice(rest, n_out, replace=False))
    role[outs] = OUTPUT
    channel[outs] = np.arange(n_out)
    return {"width": width, "height": height, "out_degree": out_degree, "long_range": long_range,
            "sigma": float(sigma), "w_std": float(w_std), "max_delay": max_delay,
            "max_draws": max_draws, "seed": int(seed), "accept": accept, "role": role,
            "sign": np.ones(n, np.int8), "channel": channel}


def grid_graph_host(spec: dict) -> SNNGraph:
    """The graph snc_b200_graph_generate_grid builds from `spec`, built on the
    host (vectorised over neurons, one draw index at a time)."""
    W, H, k, lr = spec["width"], spec["height"], spec["out_degree"], spec["long_range"]
    n, k_loc, seed = W * H, k - lr, spec["seed"]
    max_draws = spec["max_draws"] or 1000 * max(1, k)
    c_disp = np.float32(spec["sigma"] * math.sqrt(3.0) / 65536.0)
    c_w = np.float32(spec["w_std"] * math.sqrt(3.0) / 65536.0)
    accept = np.asarray(spec["accept"], np.uint32)
    posts = np.zeros((n, k), np.int32)
    got = np.zeros(n, np.int64)
    ids = np.arange(n)
    x, y = ids % W, ids // W
    d = 0
    active = ids[got < k_loc]
    while active.shape[0]:
        r = _philox(active, np.full(active.shape, d), 0, 0, seed)
        dx = np.rint(_halves_sum(r[0], r[1]).astype(np.float32) * c_disp).astype(np.int64)
        dy = np.rint(_halves_sum(r[2], r[3]).astype(np.float32) * c_disp).astype(np.int64)
        j = ((y[active] + dy) % H) * W + (x[active] + dx) % W
        u = _philox(active, np.full(active.shape, d), 1, 0, seed)[0]
        keep = (u < accept[j]) | (d >= max_draws)
        a = active[keep]
        posts[a, got[a]] = j[keep]
        got[a] += 1
        active = active[got[active] < k_loc]
        d += 1
    for q in range(lr):
        u = _philox(ids, np.full(n, q), 2, 0, seed)[0]
        posts[:, k_loc + q] = ((u.astype(np.uint64) * np.uint64(n)) >> np.uint64(32)).astype(np.int32)
    w = np.zeros((n, k), np.float32)
    dl = np.zeros((n, k), np.int32)
    for s in range(k):
        r = _philox(ids, np.full(n, s), 3, 0, seed)
        w[:, s] = _halves_sum(r[0], r[1]).astype(np.float32) * c_w
        dl[:, s] = 1 + ((r[2].astype(np.uint64) * np.uint64(spec["max_delay"])) >> np.uint64(32)).astype(np.int32)
    row_ptr = (np.arange(n + 1, dtype=np.int64) * k).astype(np.int32)
    return SNNGraph(n, row_ptr, posts.ravel(), w.ravel(), dl.ravel(), spec["role"], spec["sign"],
                    spec["channel"])
