"""ctypes binding of libsnc_b200.so (the C ABI in include/snc_b200.h).

The library is required: importing a function from here when it is missing
raises, there is no CPU fallback.  Build it with ``python -m snc_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .build import LIB, build, up_to_date

OK, EINVAL, ENODEV, ENOMEM, ECUDA, ETIMEOUT, EUNSUPPORTED, EOVERFLOW = 0, -1, -2, -3, -4, -5, -6, -7
MODE_ATOMIC, MODE_BUCKET, MODE_SORT, MODE_AUTO = 0, 1, 2, 3
PATH_PLAIN, PATH_PERSISTENT, PATH_AUTO = 0, 1, 2
RUN_RASTER, RUN_VFINAL, RUN_GRAPH, RUN_FORCE_GRID = 1, 2, 4, 8
ENCODER_DIRECT, ENCODER_POISSON, ENCODER_LATENCY = 0, 1, 2

STATUS_NAMES = {0: "OK", -1: "EINVAL", -2: "ENODEV", -3: "ENOMEM", -4: "ECUDA", -5: "ETIMEOUT",
                -6: "EUNSUPPORTED", -7: "EOVERFLOW"}


class SncB200Error(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"snc_b200 {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class GraphView(C.Structure):
    _fields_ = [("num_neurons", C.c_int32), ("num_synapses", C.c_int32),
                ("row_ptr", C.c_void_p), ("post_ids", C.c_void_p), ("weights", C.c_void_p),
                ("delays", C.c_void_p), ("role", C.c_void_p), ("sign", C.c_void_p),
                ("channel", C.c_void_p)]


class Lif(C.Structure):
    _fields_ = [("threshold", C.c_float), ("decay", C.c_float), ("reset", C.c_float),
                ("refractory", C.c_int32), ("reset_mode", C.c_int32)]


class LaunchConfig(C.Structure):
    _fields_ = [("mode", C.c_int32), ("path", C.c_int32), ("tier", C.c_int32),
                ("block_threads", C.c_int32), ("wave", C.c_int32), ("ring_smem", C.c_int32),
                ("ms", C.c_float)]


class GridGraph(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("out_degree", C.c_int32),
                ("long_range", C.c_int32), ("sigma", C.c_float), ("w_std", C.c_float),
                ("max_delay", C.c_int32), ("max_draws", C.c_int32), ("seed", C.c_uint64)]


class StructConfig(C.Structure):
    _fields_ = [("grow_per_epoch", C.c_int32), ("delay", C.c_int32), ("w_grow_init", C.c_float),
                ("locality_window", C.c_float), ("protect_rounds", C.c_int32),
                ("max_attempts_mult", C.c_int32), ("reward_modulated", C.c_int32),
                ("reward_chance", C.c_float), ("reward_floor", C.c_float)]


class StructReport(C.Structure):
    _fields_ = [("pruned", C.c_int32), ("grown", C.c_int32), ("synapses", C.c_int32)]


class RunStats(C.Structure):
    _fields_ = [("spikes", C.c_int64), ("synaptic_events", C.c_int64), ("overflow", C.c_int32),
                ("ms", C.c_double)]


# name -> (restype, argtypes); every function of include/snc_b200.h
P = C.c_void_p
I32 = C.c_int32
SIGNATURES = {
    "snc_b200_available": (C.c_int, []),
    "snc_b200_abi_version": (C.c_int, []),
    "snc_b200_set_device": (C.c_int, [C.c_int]),
    "snc_b200_inputs_info": (C.c_int, [P, P, P]),
    "snc_b200_inputs_read": (C.c_int, [P, P, P, P]),
    "snc_b200_inputs_encode": (C.c_int, [P, I32, P, I32, I32, P, C.c_float, C.c_float, C.c_float,
                                         C.c_uint64, P]),
    "snc_b200_last_error": (C.c_char_p, []),
    "snc_b200_set_wait_limit": (C.c_int, [C.c_uint64]),
    "snc_b200_inject_stall": (C.c_int, [I32]),
    "snc_b200_inject_alloc_failure": (C.c_int, [C.c_int64]),
    "snc_b200_probe_red_rate": (C.c_int, [C.c_int64, C.c_int64, P]),
    "snc_b200_connectome_layered_local": (C.c_int, [P, I32, I32, I32, C.c_float, C.c_uint64, P]),
    "snc_b200_connectome_release": (C.c_int, [P]),
    "snc_b200_connectome_info": (C.c_int, [P, P, P]),
    "snc_b200_connectome_read": (C.c_int, [P] * 6),
    "snc_b200_connectome_set_weights": (C.c_int, [P, P, C.c_int64]),
    "snc_b200_connectome_update": (C.c_int, [P, P, C.c_int64, P, C.c_float, P]),
    "snc_b200_connectome_graph": (C.c_int, [P, P]),
    "snc_b200_graph_upload": (C.c_int, [P, P]),
    "snc_b200_graph_release": (C.c_int, [P]),
    "snc_b200_graph_upload_sncg": (C.c_int, [P, C.c_size_t, P]),
    "snc_b200_graph_generate_grid": (C.c_int, [P, P, P, P, P, P]),
    "snc_b200_graph_info": (C.c_int, [P, P, P, P, P, P]),
    "snc_b200_graph_layout": (C.c_int, [P] * 11),
    "snc_b200_inputs_upload": (C.c_int, [P, P, C.c_size_t, I32, P, P]),
    "snc_b200_inputs_release": (C.c_int, [P]),
    "snc_b200_run_create": (C.c_int, [P, P, C.c_int, P]),
    "snc_b200_run_release": (C.c_int, [P]),
    "snc_b200_run_launch": (C.c_int, [P, P, C.c_int, C.c_int, P]),
    "snc_b200_run_fetch": (C.c_int, [P, P, P, P, P, P, P]),
    "snc_b200_run_used": (C.c_int, [P, P, P]),
    "snc_b200_run_used_graph": (C.c_int, [P]),
    "snc_b200_forward": (C.c_int, [P, P, P, C.c_size_t, I32, P, C.c_int, P, P]),
    "snc_b200_forward_batched": (C.c_int, [P, P, C.c_size_t, I32, P, P, C.c_int, P, P, P, P]),
    "snc_b200_autotune": (C.c_int, [P, P, P, P, P, P]),
    "snc_b200_autotune_ex": (C.c_int, [P, P, P, P, I32, P, P]),
    "snc_b200_autotune_lookup": (C.c_int, [P, P, P]),
    "snc_b200_run_configure": (C.c_int, [P, P]),
    "snc_b200_part_create": (C.c_int, [P, P, I32, I32, P, P]),
    "snc_b200_part_release": (C.c_int, [P]),
    "snc_b200_part_integrate": (C.c_int, [P, I32, P, P]),
    "snc_b200_part_deliver": (C.c_int, [P, I32, P, P]),
    "snc_b200_part_fetch": (C.c_int, [P, P, P, P, P, P]),
    "snc_b200_run_set_readout": (C.c_int, [P, C.c_float]),
    "snc_b200_eprop_create": (C.c_int, [P, P, P, I32, P, P, P]),
    "snc_b200_eprop_release": (C.c_int, [P]),
    "snc_b200_eprop_path": (C.c_int, [P]),
    "snc_b200_eprop_set_weights": (C.c_int, [P, P]),
    "snc_b200_eprop_get_weights": (C.c_int, [P, P]),
    "snc_b200_eprop_batch": (C.c_int, [P, P, C.c_size_t, I32, P, P, C.c_int, P, P]),
    "snc_b200_eprop_get_eligibility": (C.c_int, [P, P]),
    "snc_b200_eprop_gradient": (C.c_int, [P, P, C.c_size_t, I32, P, P, P, P, P]),
    "snc_b200_eprop_apply": (C.c_int, [P, P, I32]),
    "snc_b200_eprop_reset_stats": (C.c_int, [P]),
    "snc_b200_eprop_collect_stats": (C.c_int, [P, P, P]),
    "snc_b200_bptt_create": (C.c_int, [I32, I32, P, P, P, P]),
    "snc_b200_bptt_release": (C.c_int, [P]),
    "snc_b200_bptt_set_resident": (C.c_int, [P, I32]),
    "snc_b200_bptt_forward": (C.c_int, [P, P, P, I32, I32, C.c_float, C.c_float, C.c_float, I32,
                                        I32, P, P, P, P]),
    "snc_b200_bptt_backward": (C.c_int, [P, P, P, I32, I32, C.c_float, C.c_float, C.c_float, I32,
                                         I32, P, P, P, P, P, P, P]),
    "snc_b200_leaky_scan": (C.c_int, [P, P, I32, C.c_int64, C.c_float, I32, P]),
    "snc_b200_transpose": (C.c_int, [P, P, I32, I32, I32, C.c_int64, C.c_int64, P]),
    "snc_b200_bptt_forward_static": (C.c_int, [P, P, P, I32, I32, C.c_float, C.c_float, C.c_float,
                                               I32, I32, P, P, P, P]),
}

_LIB = None


def lib():
    """The loaded library.  Raises when it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB):
            raise ImportError(f"{LIB} is missing: build it with `python -m snc_b200.build`")
        if not up_to_date():
            build()
        L = C.CDLL(LIB)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(rc: int, what: str = "") -> None:
    if rc != OK:
        msg = lib().snc_b200_last_error().decode(errors="replace")
        raise SncB200Error(rc, f"{what}: {msg}" if what else msg)


def ptr(a) -> int | None:
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return a.ctypes.data
    return a
