"""snc_b200_inputs_encode -- the encoders run on the device -- against the
CPU restatement (oracle/encoders.py, itself pinned to the reference's
encode() and to Philox's known answers): the schedule read back is bit-for-bit
the schedule of the restated events, for direct, latency and Poisson, with a
threshold, uneven and zero step counts and channels driving several input
neurons; a forward on the encoded batch equals a forward on the uploaded
events."""
import numpy as np
import pytest

from oracle import encoders as E
from oracle import oracle as O
from snc_b200 import runtime as R
from tests.helpers import input_graph

pytestmark = pytest.mark.gpu


def _check(g, f, steps, enc, **kw):
    dg = R.DeviceGraph(g)
    di = R.DeviceInputs.encode(dg, f, steps, encoder=enc, **kw)
    ptr, nid, ext = di.read()
    ev = E.encode_batch(R.DeviceInputs.ENCODERS[enc], f, steps, **kw)
    base = 0
    for b, T in enumerate(steps):
        optr, onid, oext = O.schedule_merged(g, ev, b, int(T))
        p = ptr[base + b: base + b + T + 1]
        assert np.array_equal(p - p[0], optr), f"{enc} sample {b}: step pointers"
        assert np.array_equal(nid[p[0]:p[-1]], onid), f"{enc} sample {b}: neurons"
        assert np.array_equal(ext[p[0]:p[-1]].view(np.uint32), oext.view(np.uint32)), \
            f"{enc} sample {b}: drive bits"
        base += int(T)
    return dg, di, ev


@pytest.mark.parametrize("enc", ["direct", "latency", "poisson"])
@pytest.mark.parametrize("fan", [1, 3])
def test_encoded_schedule_matches_restatement(enc, fan):
    g = input_graph(60, fan=fan, seed=fan)
    n_ch = 60 // fan + 2  # two channels without input neurons
    rng = np.random.default_rng(9)
    f = rng.random((5, n_ch), dtype=np.float32) * np.float32(1.2)
    f[:, ::5] = 0.0
    steps = [37, 0, 120, 1, 64]
    dg, di, _ = _check(g, f, steps, enc, gain=1.25, max_rate=0.4, threshold=0.1, seed=77)
    di.release()
    dg.release()


def test_forward_on_encoded_batch_equals_uploaded_events():
    g = input_graph(200, n_hid=300, seed=4)
    rng = np.random.default_rng(2)
    f = rng.random((6, 200), dtype=np.float32)
    steps = np.array([50, 80, 20, 65, 0, 33], np.int32)
    dg, di, ev = _check(g, f, steps, "poisson", gain=2.0, max_rate=0.3, seed=5)
    lif = R.LIFParams(threshold=1.0, decay=0.9, reset=0.0, refractory=1, reset_mode=0)
    r1 = R.Run(dg, di, raster=True)
    r1.launch(lif, mode=R.MODE_SORT, path=R.PATH_PERSISTENT)
    a = r1.fetch(raster=True)
    di2 = R.DeviceInputs(dg, ev, steps)
    r2 = R.Run(dg, di2, raster=True)
    r2.launch(lif, mode=R.MODE_SORT, path=R.PATH_PERSISTENT)
    b = r2.fetch(raster=True)
    assert a["total_spikes"] > 0
    assert np.array_equal(a["raster"], b["raster"]) and np.array_equal(a["logits"], b["logits"])
    for x in (r1, r2, di, di2, dg):
        x.release()


def test_encode_rejects_bad_arguments():
    g = input_graph(10)
    dg = R.DeviceGraph(g)
    with pytest.raises(Exception):
        R.DeviceInputs.encode(dg, np.ones((2, 10), np.float32), [5, 5], encoder=7)
    with pytest.raises(Exception):
        R.DeviceInputs.encode(dg, np.ones((2, 10), np.float32), [5, -1])
    dg.release()
