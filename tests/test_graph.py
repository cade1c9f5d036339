"""Host graph type, the SNCG wire format and the benchmark workloads."""
import os
import subprocess

import numpy as np
import pytest

from oracle import REF_ROOT
from oracle import oracle as O
from snc_b200 import graph as G
from snc_b200 import workloads as W

REF_EXPORT = os.path.join(os.path.dirname(O.__file__), "_ref", "snc_export")


def test_sncg_round_trip(tmp_path):
    g = W.random_graph(7, max_delay=6)
    p = tmp_path / "g.bin"
    G.save_sncg(g, p)
    d = G.load_graph(p)
    assert d["N"] == g.num_neurons and d["S"] == g.num_synapses
    np.testing.assert_array_equal(d["pre"], g.pre_ids())
    np.testing.assert_array_equal(d["post"], g.post_ids)
    h = G.graph_from_sncg(d)
    for k in ("row_ptr", "post_ids", "weights", "delays", "role", "sign", "channel"):
        np.testing.assert_array_equal(getattr(h, k), getattr(g, k))
    G.save_sncg(g, p, with_weights=False)
    d2 = G.load_graph(p)
    assert "weights" not in d2


@pytest.mark.skipif(not os.path.exists(REF_EXPORT), reason="reference snc_export not built")
def test_reads_reference_snc_export_output(tmp_path):
    """The reference exporter (src/bench/snc_export.cpp) writes the file; our
    loader returns the same dict as python/snc/graph.py would."""
    p = tmp_path / "ref.bin"
    subprocess.check_call([REF_EXPORT, "--structure", "static-snc", "--layers", "784,256,10",
                           "--synapse-budget", "40000", "--seed", "3", "--delay-max", "4",
                           "--out", str(p)], stdout=subprocess.DEVNULL)
    d = G.load_graph(p)
    ref = O.ref_generate("static-snc", [784, 256, 10], synapse_budget=40000, weight=0.5,
                         delay=1, inhib=0.2, seed=3)
    assert d["N"] == ref.num_neurons and d["S"] == ref.num_synapses
    np.testing.assert_array_equal(d["pre"], ref.pre_ids())
    np.testing.assert_array_equal(d["post"], ref.post_ids)
    assert d["delays"].min() >= 1 and d["delays"].max() <= 4
    g = G.graph_from_sncg(d)
    assert g.validate() == ""
    assert g.num_input_channels == d["n_in"] == 784 and g.num_output_channels == d["n_out"] == 10
    ref_loader = os.path.join(REF_ROOT, "python", "snc", "graph.py")
    if os.path.exists(ref_loader):
        import importlib.util
        spec = importlib.util.spec_from_file_location("ref_graph", ref_loader)
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        rd = m.load_graph(str(p))
        for k in ("N", "S", "n_in", "n_out"):
            assert rd[k] == d[k]
        for k in ("pre", "post", "delays", "role", "channel"):
            np.testing.assert_array_equal(rd[k], d[k])


def test_bad_magic(tmp_path):
    p = tmp_path / "x.bin"
    np.array([1, 2, 3, 4, 5], dtype="<i4").tofile(p)
    with pytest.raises(ValueError):
        G.load_graph(p)


def test_validate_matches_reference_rules():
    g = W.random_graph(1)
    assert g.validate() == ""
    g.delays = g.delays.copy()
    g.delays[0] = 0
    assert g.validate() == "delay < 1"


def test_workloads_deterministic_and_shaped():
    a, b = W.ff784_graph(seed=1), W.ff784_graph(seed=1)
    np.testing.assert_array_equal(a.post_ids, b.post_ids)
    np.testing.assert_array_equal(a.weights, b.weights)
    assert a.num_neurons == 1050 and a.num_synapses == 256 * 32 + 10 * 32
    fi = np.bincount(a.post_ids, minlength=a.num_neurons)
    assert (fi[784:] == 32).all()
    assert a.delays.min() >= 1 and a.delays.max() <= 4
    ev, steps = W.ff784_inputs(3, 50)
    assert set(np.unique(ev["sample_id"])) == {0, 1, 2} and (steps == 50).all()
    g3 = W.audio700_graph()
    assert g3.num_input_channels == 700 and g3.num_output_channels == 20
    assert g3.max_delay == 30
    ev3, st3 = W.audio700_inputs(6)
    assert st3.min() >= 50 and st3.max() <= 1000


@pytest.mark.slow
def test_rec100k_shape():
    g = W.rec100k_graph()
    s = g.stats()
    assert s["num_neurons"] == 100_000 and s["num_synapses"] == 10_000_000
    assert s["fan_in_cv"] > 0.9  # heavy-tailed in-degree
    assert g.max_delay == 30 and g.num_input_channels == 10_000


def test_sncg_device_ingest_rejects_bad_headers_on_the_host(tmp_path):
    """snc_b200_graph_upload_sncg checks the header, the sizes and the
    per-neuron arrays on the host before touching a device."""
    import ctypes as C
    from snc_b200 import _lib
    g = W.random_graph(2)
    p = tmp_path / "g.sncg"
    G.save_sncg(g, p)
    data = bytearray(p.read_bytes())
    L = _lib.lib()

    def status(b):
        h = C.c_void_p()
        buf = (C.c_char * len(b)).from_buffer_copy(bytes(b))
        return L.snc_b200_graph_upload_sncg(buf, len(b), C.byref(h))

    bad = bytearray(data); bad[0] ^= 1
    assert status(bad) == _lib.EINVAL and "magic" in L.snc_b200_last_error().decode()
    assert status(data[:len(data) // 2]) == _lib.EINVAL
    assert "truncated" in L.snc_b200_last_error().decode()
    assert status(data[:12]) == _lib.EINVAL
    N, S = g.num_neurons, g.num_synapses
    words = np.frombuffer(bytes(data), dtype="<i4").copy()
    words[5 + 3 * S + 1] = 7  # a role outside 0..2
    assert status(words.tobytes()) == _lib.EINVAL and "role" in L.snc_b200_last_error().decode()
