"""CPU restatement of the post-neuron partitioned forward.  TEST
INFRASTRUCTURE ONLY: the checker of snc_b200.parallel.PartitionedForward and
of snc_b200_part_* (one sample).

One rank owns neurons [lo, hi): their membrane potential, refractory count
and delay-ring columns.  Per step it integrates its neurons exactly as the
serial CPU backend does (src/runtime/cpu_backend.cpp:129-143, drive summed in
event order, :99), exchanges its spike bits through `gather` (every rank
receives all N bits), then adds the synapses of every fired neuron, in
ascending pre id and CSR edge order, whose post it owns
(cpu_backend.cpp:172-181 restricted to its columns).  Every ring cell has one
owner and receives its contributions in the CPU order, so the ranks' results
together equal the single-process forward bit for bit."""
from __future__ import annotations

import numpy as np

from . import oracle as O


def partition_forward(g, events, T, lif, lo, hi, gather):
    """This rank's part of one sample's forward.  gather(bool[hi - lo]) ->
    bool[N] (the spike bits of every rank, in neuron order).  Returns
    dict(raster [T][ceil(N/32)] with this rank's bits, v [hi - lo], spikes,
    events, logits [n_out])."""
    N = g.num_neurons
    R = int(np.max(g.delays)) + 1 if g.num_synapses else 2
    Wd = (N + 31) // 32
    rp, post = np.asarray(g.row_ptr), np.asarray(g.post_ids)
    w = np.asarray(g.weights, np.float32)
    delays = np.asarray(g.delays)
    sign = np.asarray(g.sign, np.float32)
    role, ch = np.asarray(g.role), np.asarray(g.channel)
    sp, nid, ext_v = O.schedule_merged(g, events, 0, T)
    v = np.zeros(hi - lo, np.float32)
    refr = np.zeros(hi - lo, np.int32)
    ring = np.zeros((R, N), np.float32)
    raster = np.zeros((T, Wd), np.uint32)
    noc = max(1, g.num_output_channels)
    logits = np.zeros(noc, np.float32)
    spikes = events_n = 0
    decay, thr = np.float32(lif.decay), np.float32(lif.threshold)
    for t in range(T):
        slot = t % R
        ext = np.zeros(hi - lo, np.float32)
        for k in range(sp[t], sp[t + 1]):
            if lo <= nid[k] < hi:
                ext[nid[k] - lo] = ext_v[k]
        rin = ring[slot, lo:hi].copy()
        ring[slot, lo:hi] = 0.0
        fired = np.zeros(hi - lo, bool)
        for q in range(hi - lo):
            if refr[q] > 0:
                refr[q] -= 1
                v[q] = np.float32(lif.reset)
                continue
            nv = np.float32(np.float32(np.float32(v[q] * decay) + ext[q]) + rin[q])
            if nv >= thr:
                v[q] = np.float32(nv - thr) if lif.reset_mode == 1 else np.float32(lif.reset)
                refr[q] = lif.refractory
                fired[q] = True
            else:
                v[q] = nv
        own = np.nonzero(fired)[0] + lo
        spikes += own.shape[0]
        for i in own:
            events_n += int(rp[i + 1] - rp[i])
            raster[t, i >> 5] |= np.uint32(1 << (i & 31))
            if role[i] == 2 and ch[i] >= 0:
                logits[ch[i]] += 1.0
        all_fired = gather(fired)
        for i in np.nonzero(all_fired)[0]:
            s = sign[i]
            for e in range(rp[i], rp[i + 1]):
                p = post[e]
                if lo <= p < hi:
                    c = (t + delays[e]) % R
                    ring[c, p] = np.float32(ring[c, p] + np.float32(s * w[e]))
    return {"raster": raster, "v": v, "spikes": spikes, "events": events_n,
            "logits": logits[:g.num_output_channels]}
