"""ctypes binding of include/rtdsl.h.

The library is the product: there is no CPU fallback.  If librtdsl.so is
missing and cannot be built, importing the binding raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

from . import _build

RTD_OK = 0
RTD_ERR_INVALID_ARGUMENT = 1
RTD_ERR_CUDA = 2
RTD_ERR_OUT_OF_MEMORY = 3
RTD_ERR_OVERFLOW = 4
RTD_ERR_NOT_CONVERGED = 5
RTD_ERR_TIMEOUT = 6
RTD_ERR_UNSUPPORTED = 7
RTD_ERR_NO_DEVICE = 8

RADIUS_SAMPLED_NN = 0
RADIUS_SAMPLED_PERCENTILE = 1
RADIUS_FIXED = 2
RADIUS_SAMPLED_MAX = 3
RADIUS_MORTON_WINDOW = 4

EMPTY_ID = 0xFFFFFFFF


class RtdError(RuntimeError):
    """A C-ABI call returned a status other than RTD_OK."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_status_name(status)}: {message}")
        self.status = status


class Schedule(C.Structure):
    """rtd_schedule: gprt-ir Schedule (gprt-ir/src/lib.rs:58-89) re-expressed."""
    _fields_ = [
        ("radius_increment_mult", C.c_float),
        ("max_rounds", C.c_uint32),
        ("radius_heuristic", C.c_int32),
        ("radius_param", C.c_float),
        ("use_morton_lbv", C.c_uint32),
        ("leaf_size", C.c_uint32),
        ("block_size", C.c_uint32),
        ("lanes_per_query", C.c_uint32),
        ("morton_bits", C.c_uint32),
        ("partial_results", C.c_uint32), ("reserved", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class IndexInfo(C.Structure):
    _fields_ = [
        ("n_points", C.c_uint64),
        ("n_internal", C.c_uint64),
        ("leaf_size", C.c_uint32),
        ("morton_bits", C.c_uint32),
        ("lo", C.c_float * 3),
        ("hi", C.c_float * 3),
    ]


_P = C.c_void_p
_U64 = C.c_uint64
_U32 = C.c_uint32
_F = C.c_float
_I = C.c_int

# name -> (restype, argtypes); mirrors include/rtdsl.h
_SIGNATURES = {
    "rtd_schedule_default": (None, [C.POINTER(Schedule)]),
    "rtd_status_string": (C.c_char_p, [_I]),
    "rtd_last_error": (C.c_char_p, []),
    "rtd_version": (_I, []),
    "rtd_index_create": (_I, [C.POINTER(_P)]),
    "rtd_index_destroy": (_I, [_P]),
    "rtd_index_build": (_I, [_P, _P, _U64, C.POINTER(Schedule), _P]),
    "rtd_index_info_get": (_I, [_P, C.POINTER(IndexInfo), _P]),
    "rtd_knn": (_I, [_P, _P, _U64, _U32, C.POINTER(Schedule), _P, _P, _P]),
    "rtd_k_nn": (_I, [_P, _P, _U64, _P, _U64, _U32, C.POINTER(Schedule), _P, _P, _P]),
    "rtd_knn_graph_create": (_I, [_P, _U64, _P, _U64, _U32, C.POINTER(Schedule), _P, _P, _P,
                                  C.POINTER(_P)]),
    "rtd_knn_graph_create_host": (_I, [_P, _U64, _P, _U64, _U32, C.POINTER(Schedule), _P, _P,
                                       C.POINTER(_P)]),
    "rtd_knn_graph_launch": (_I, [_P, _P]),
    "rtd_knn_graph_errors": (_I, [_P, _P]),
    "rtd_knn_graph_destroy": (_I, [_P]),
    "rtd_context_create": (_I, [C.POINTER(_P)]),
    "rtd_context_destroy": (_I, [_P]),
    "rtd_k_nn_host": (_I, [_P, _P, _U64, _P, _U64, _U32, C.POINTER(Schedule), _P, _P]),
    "rtd_range_count": (_I, [_P, _P, _U64, _F, C.POINTER(Schedule), _P, C.POINTER(_U64), _P]),
    "rtd_range_fill": (_I, [_P, _P, _U64, _F, C.POINTER(Schedule), _P, _U64, _I,
                            C.POINTER(_U64), _P]),
    "rtd_range_query_host": (_I, [_P, _P, _U64, _P, _U64, _F, _P, _U64, C.POINTER(_U64)]),
    "rtd_dbscan": (_I, [_P, _P, _U64, _F, _U32, _P, C.POINTER(_U64), _P]),
    "rtd_load_points_csv": (_I, [C.c_char_p, _P, _U64, C.POINTER(_U64)]),
    "rtd_knn_backward": (_I, [_P, _U64, _P, _U64, _U32, _P, _P, _P, _P, _P]),
    "rtd_index_profile_enable": (_I, [_P, _I]),
    "rtd_index_profile_get": (_I, [_P, _P]),
    "rtd_launch_count": (_U64, []),
    "rtd_wait_selftest": (_I, [_U32, _I, _P]),
    "rtd_radix_sort_pairs": (_I, [_P, _U32, _P, _U64, _U32, _P]),
    "rtd_exclusive_scan": (_I, [_P, _P, _P, _U64, _P, _P]),
    "rtd_limits_set": (_I, [_P]),
    "rtd_limits_get": (None, [_P]),
    "rtd_bh_params_default": (None, [_P]),
    "rtd_bh_create": (_I, [C.POINTER(_P)]),
    "rtd_bh_destroy": (_I, [_P]),
    "rtd_bh_build": (_I, [_P, _P, _P, _U64, _P, _P]),
    "rtd_bh_release": (_I, [_P]),
    "rtd_bh_forward": (_I, [_P, _P, _P, _P, _P]),
    "rtd_bh_forward_noalloc": (_I, [_P, _P, _P, _P, _P]),
    "rtd_bh_backward": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "rtd_bh_info_get": (_I, [_P, _P, _P]),
    "rtd_bh_leapfrog": (_I, [_P, _P, _P, _P, _P, _U64, _F, _U32, _P, _I, _P]),
    "rtd_bh_interaction_counts": (_I, [_P, _F, _U64, C.POINTER(_U64), C.POINTER(_U64),
                                       C.POINTER(_U64), _P]),
    "rtd_bh_export": (_I, [_P, _P, _P, _P]),
    "rtd_barnes_hut_host": (_I, [_P, _P, _U64, _F, _F, _P]),
    "rtd_batch_create": (_I, [C.POINTER(_P)]),
    "rtd_batch_destroy": (_I, [_P]),
    "rtd_batch_plan": (_I, [_P, _P, _U32, C.POINTER(Schedule)]),
    "rtd_batch_schedule_default": (None, [C.POINTER(Schedule)]),
    "rtd_knn_batched": (_I, [_P, _P, _P, _P, _P, _I, _P]),
    "rtd_knn_batched_backward": (_I, [_P, _P, _P, _P, _P, _P, _P, _P]),
}


class Cloud(C.Structure):
    """rtd_cloud: one cloud of a packed batch."""
    _fields_ = [("point_offset", C.c_uint64), ("query_offset", C.c_uint64),
                ("out_offset", C.c_uint64), ("n_points", C.c_uint32),
                ("n_queries", C.c_uint32), ("k", C.c_uint32), ("pad", C.c_uint32)]

BH_LAW_REFERENCE = 0
BH_LAW_PLUMMER = 1


class BhParams(C.Structure):
    """rtd_bh_params."""
    _fields_ = [("theta", C.c_float), ("G", C.c_float), ("eps", C.c_float), ("law", C.c_int32),
                ("quadrupole", C.c_int32), ("bucket", C.c_uint32), ("min_width", C.c_float)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class BhInfo(C.Structure):
    _fields_ = [("n_bodies", C.c_uint64), ("n_nodes", C.c_uint64), ("n_leaves", C.c_uint64),
                ("depth", C.c_uint32), ("root_min", C.c_float * 3), ("root_max", C.c_float * 3),
                ("max_stack", C.c_uint32), ("log_pages", C.c_uint32)]


class Limits(C.Structure):
    """rtd_limits: process-wide bounds of bounded device loops."""
    _fields_ = [("bh_stack_entries", C.c_uint32), ("reserved", C.c_uint32 * 7)]


def default_bh_params(**overrides) -> BhParams:
    p = BhParams()
    load().rtd_bh_params_default(C.byref(p))
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(f"unknown bh parameter {k}")
        setattr(p, k, v)
    return p


class Profile(C.Structure):
    _fields_ = [("build_sort_ms", C.c_float), ("build_tree_ms", C.c_float),
                ("seed_ms", C.c_float), ("order_ms", C.c_float), ("search_ms", C.c_float)]

    def as_dict(self) -> dict:
        return {name: float(getattr(self, name)) for name, _ in self._fields_}

_lock = threading.Lock()
_lib = None


def _status_name(s: int) -> str:
    names = {0: "RTD_OK", 1: "RTD_ERR_INVALID_ARGUMENT", 2: "RTD_ERR_CUDA",
             3: "RTD_ERR_OUT_OF_MEMORY", 4: "RTD_ERR_OVERFLOW", 5: "RTD_ERR_NOT_CONVERGED",
             6: "RTD_ERR_TIMEOUT", 7: "RTD_ERR_UNSUPPORTED", 8: "RTD_ERR_NO_DEVICE"}
    return names.get(s, f"status {s}")


def declared_symbols() -> list[str]:
    return list(_SIGNATURES)


def load(build_if_missing: bool = True) -> C.CDLL:
    """Load librtdsl.so, building it first if it is missing or stale."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIB_PATH
        if build_if_missing and _build.is_stale():
            _build.build()
        if not os.path.exists(path):
            raise ImportError(f"librtdsl.so not found at {path}; run rtdsl._build.build()")
        lib = C.CDLL(path, mode=C.RTLD_GLOBAL)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def check(status: int) -> None:
    if status != RTD_OK:
        msg = load().rtd_last_error().decode(errors="replace")
        raise RtdError(status, msg)


def default_batch_schedule(**overrides) -> Schedule:
    """rtd_batch_schedule_default with keyword overrides."""
    s = Schedule()
    load().rtd_batch_schedule_default(C.byref(s))
    for k, v in overrides.items():
        if not hasattr(s, k):
            raise AttributeError(f"unknown schedule field {k}")
        setattr(s, k, v)
    return s


def default_schedule(**overrides) -> Schedule:
    s = Schedule()
    load().rtd_schedule_default(C.byref(s))
    for k, v in overrides.items():
        if not hasattr(s, k):
            raise AttributeError(f"unknown schedule field {k}")
        setattr(s, k, v)
    return s
