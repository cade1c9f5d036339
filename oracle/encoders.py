"""CPU restatement of the input encoders (TEST INFRASTRUCTURE ONLY).

snc::encode (src/training/encoders.cpp:25-71) for a batch, in the form the
device encoder (snc_b200_inputs_encode) implements:
  * direct  -- every step, amplitude v * gain, for channels with v > threshold
               (encoders.cpp:32-41): identical to the reference;
  * latency -- one spike of amplitude gain at t = lround((T-1) * (1 - min(1, v)))
               clamped to [0, T) (encoders.cpp:56-66): identical to the reference;
  * poisson -- a spike of amplitude gain when u < min(1, v * max_rate)
               (encoders.cpp:43-54), with u drawn by Philox-4x32-10 (Salmon,
               Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2,
               3", SC 2011) instead of the reference's mt19937_64 stream: the
               same distribution, not the same draws.  Counter (t / 4, channel,
               sample, 0), key (seed low 32 bits, seed high 32 bits); output
               word t % 4 gives u = (word >> 8) * 2^-24.
Events come per sample, channel-major then step, like the reference's
concatenated per-sample encode() output.
"""
from __future__ import annotations

import numpy as np

from snc_b200.graph import EVENT_DTYPE

DIRECT, POISSON, LATENCY = 0, 1, 2

_M0, _M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
_W0, _W1 = np.uint32(0x9E3779B9), np.uint32(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr, key):
    """Philox-4x32 with 10 rounds on arrays: ctr [..., 4] uint32, key [..., 2]
    uint32 (broadcast); returns [..., 4] uint32."""
    c = [np.asarray(ctr[..., i], dtype=np.uint64) for i in range(4)]
    k0 = np.asarray(key[..., 0], dtype=np.uint32).copy()
    k1 = np.asarray(key[..., 1], dtype=np.uint32).copy()
    for _ in range(10):
        p0 = _M0 * c[0]
        p1 = _M1 * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK
        c = [(hi1 ^ c[1] ^ k0.astype(np.uint64)) & _MASK, lo1,
             (hi0 ^ c[3] ^ k1.astype(np.uint64)) & _MASK, lo0]
        with np.errstate(over="ignore"):
            k0 = k0 + _W0
            k1 = k1 + _W1
    return np.stack([x.astype(np.uint32) for x in c], axis=-1)


def poisson_uniforms(seed: int, sample: int, channel: int, T: int) -> np.ndarray:
    """The T uniforms in [0, 1) of one (sample, channel) stream."""
    nq = (T + 3) // 4
    ctr = np.zeros((nq, 4), np.uint32)
    ctr[:, 0] = np.arange(nq, dtype=np.uint32)
    ctr[:, 1] = channel
    ctr[:, 2] = sample
    key = np.array([seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF], np.uint32)
    words = philox4x32_10(ctr, key).reshape(-1)[:T]
    return (words >> np.uint32(8)).astype(np.float32) * np.float32(1.0 / 16777216.0)


def encode_batch(encoder: int, features, steps, gain=1.0, max_rate=0.5, threshold=0.0,
                 seed=1) -> np.ndarray:
    """Events of a batch: features [B, C] float32, steps [B]."""
    f = np.ascontiguousarray(features, dtype=np.float32)
    B, C = f.shape
    steps = np.asarray(steps, dtype=np.int64).reshape(B)
    gain, max_rate, threshold = np.float32(gain), np.float32(max_rate), np.float32(threshold)
    rows = []
    for b in range(B):
        T = int(steps[b])
        for c in range(C):
            v = f[b, c]
            if not v > threshold:
                continue
            if encoder == DIRECT:
                ts = np.arange(T)
                amp = np.float32(v * gain)
            elif encoder == LATENCY:
                if T <= 0:
                    continue
                vc = min(np.float32(1.0), v)
                x = np.float32(np.float32(T - 1) * np.float32(np.float32(1.0) - vc))
                t = int(np.floor(np.float64(x) + 0.5))  # lround, x >= 0 (exact in double)
                ts = np.array([min(max(t, 0), T - 1)])
                amp = gain
            else:
                prob = min(np.float32(1.0), np.float32(v * max_rate))
                u = poisson_uniforms(seed, b, c, T)
                ts = np.nonzero(u < prob)[0]
                amp = gain
            if ts.size:
                e = np.zeros(ts.size, dtype=EVENT_DTYPE)
                e["sample_id"] = b
                e["channel_id"] = c
                e["time"] = ts
                e["amplitude"] = amp
                rows.append(e)
    return np.concatenate(rows) if rows else np.zeros(0, dtype=EVENT_DTYPE)
