"""The C ABI library without a GPU: it loads, exports every function that
include/snc_b200.h declares, and rejects invalid graphs before touching a
device (the checks of SNNGraph::validate, src/graph/snn_graph.cpp:30-56)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from snc_b200 import _lib
from snc_b200 import runtime as R
from snc_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(snc_b200_\w+)\s*\(", text)))


def test_library_loads_and_exports_every_declared_symbol():
    L = _lib.lib()
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            names += declared(h)
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.snc_b200_abi_version() == 1


def test_python_signatures_cover_the_header():
    assert set(declared("snc_b200.h")) <= set(_lib.SIGNATURES)


def _graph_status(g):
    view = R.graph_view(g)
    h = C.c_void_p()
    return _lib.lib().snc_b200_graph_upload(C.byref(view), C.byref(h)), h


def test_invalid_graphs_are_rejected_without_a_device():
    g = W.random_graph(1)
    bad = W.random_graph(1)
    bad.delays = bad.delays.copy()
    bad.delays[3] = 0
    assert _graph_status(bad)[0] == _lib.EINVAL
    bad = W.random_graph(1)
    bad.post_ids = bad.post_ids.copy()
    bad.post_ids[0] = g.num_neurons
    assert _graph_status(bad)[0] == _lib.EINVAL
    bad = W.random_graph(1)
    bad.row_ptr = bad.row_ptr.copy()
    bad.row_ptr[5], bad.row_ptr[6] = bad.row_ptr[6] + 1, bad.row_ptr[5]
    assert _graph_status(bad)[0] == _lib.EINVAL
    big = W.random_graph(1)
    big.delays = big.delays.copy()
    big.delays[0] = 300
    assert _graph_status(big)[0] == _lib.EUNSUPPORTED


@pytest.mark.skipif(os.environ.get("CUDA_VISIBLE_DEVICES", None) is None and
                    __import__("torch").cuda.is_available(), reason="a GPU is present")
def test_valid_graph_without_device_reports_enodev():
    rc, _ = _graph_status(W.random_graph(1))
    if rc == _lib.OK:
        pytest.skip("a device is present")
    assert rc == _lib.ENODEV
    assert "device" in _lib.lib().snc_b200_last_error().decode()
    assert R.available() is False


def test_backend_names():
    assert R.parse_backend("cuda-sort") == _lib.MODE_SORT
    assert R.parse_backend("cuda-atomic") == _lib.MODE_ATOMIC
    assert R.parse_backend("b200-bucket") == _lib.MODE_BUCKET
    assert R.backend_name(_lib.MODE_SORT) == "b200-sort"
    with pytest.raises(ValueError):
        R.parse_backend("cpu")


def test_event_layout_matches_c_struct():
    from snc_b200.graph import EVENT_DTYPE
    assert EVENT_DTYPE.itemsize == 16
    assert [EVENT_DTYPE.fields[k][1] for k in ("sample_id", "channel_id", "time", "amplitude")] == [0, 4, 8, 12]
    assert C.sizeof(_lib.Lif) == 20 and C.sizeof(_lib.RunStats) == 32
    assert C.sizeof(_lib.GraphView) == 8 + 7 * 8
    assert np.dtype(np.float32).itemsize == 4
