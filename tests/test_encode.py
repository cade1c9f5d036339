"""The CPU restatement of the input encoders (oracle/encoders.py), pinned:
Philox-4x32-10 against the known-answer vectors published with the
algorithm's reference implementation (Random123), direct and latency
against the reference's own encode() event for event, and the Poisson rule's
spike rate against its expectation and against the reference encoder."""
import numpy as np
import pytest

from oracle import encoders as E
from oracle import oracle as O


@pytest.mark.parametrize("ctr,key,want", [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
])
def test_philox_known_answers(ctr, key, want):
    got = E.philox4x32_10(np.array([ctr], np.uint32), np.array([key], np.uint32))[0]
    assert [int(x) for x in got] == want


@pytest.mark.skipif(not O.ref_available(), reason="reference build missing (oracle/Makefile ref)")
@pytest.mark.parametrize("enc,name", [(E.DIRECT, "direct"), (E.LATENCY, "latency")])
def test_exact_encoders_match_reference(enc, name):
    rng = np.random.default_rng(3)
    f = rng.random((4, 60), dtype=np.float32) * np.float32(1.3)
    f[:, ::7] = 0.0
    f[1, 3] = 0.05  # == threshold: dropped
    steps = [40, 13, 1, 7]
    got = E.encode_batch(enc, f, steps, gain=1.5, max_rate=0.3, threshold=0.05)
    ref = np.concatenate([O.ref_encode(name, f[b], steps[b], gain=1.5, max_rate=0.3,
                                       threshold=0.05, sample_id=b) for b in range(4)])
    assert np.array_equal(got, ref)


def test_poisson_rate():
    f = np.full((2, 100), 0.5, np.float32)
    ev = E.encode_batch(E.POISSON, f, [1500, 1500], max_rate=0.2, seed=11)
    n = 2 * 100 * 1500
    p = 0.1
    assert abs(len(ev) / n - p) < 5 * np.sqrt(p * (1 - p) / n)
    # per channel, and the two samples draw different streams
    per = np.bincount(ev["channel_id"] + 100 * ev["sample_id"], minlength=200)
    assert abs(per.mean() - 150) < 5 and per.std() < 3 * np.sqrt(150)
    a = ev[ev["sample_id"] == 0]
    b = ev[ev["sample_id"] == 1]
    assert not np.array_equal(a[["channel_id", "time"]], b[["channel_id", "time"]])
    assert np.array_equal(E.encode_batch(E.POISSON, f, [1500, 1500], max_rate=0.2, seed=11), ev)


@pytest.mark.skipif(not O.ref_available(), reason="reference build missing (oracle/Makefile ref)")
def test_poisson_rate_matches_reference():
    rng = np.random.default_rng(4)
    f = rng.random((1, 300), dtype=np.float32)
    ours = E.encode_batch(E.POISSON, f, [800], max_rate=0.25, seed=3)
    ref = O.ref_encode("poisson", f[0], 800, max_rate=0.25, seed=3)
    expect = float(np.minimum(1.0, f[0] * np.float32(0.25)).sum()) * 800
    for n in (len(ours), len(ref)):
        assert abs(n - expect) < 5 * np.sqrt(expect)
