"""ctypes binding of the C ABI declared in include/nwgrad_b200.h.

The shared library is the product's only compute path: if it is missing or fails to load,
every call raises (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)
_u16p = C.POINTER(C.c_uint16)

NWG_OK, NWG_EINVAL, NWG_ECUDA, NWG_ENOMEM, NWG_ESTATE, NWG_ERANGE = range(6)


class Job(C.Structure):
    _fields_ = [("gap_model", C.c_int), ("mode", C.c_int), ("grad_mode", C.c_int),
                ("precision", C.c_int), ("band", C.c_int), ("keep_paths", C.c_int),
                ("temperature", C.c_double), ("soft_double", C.c_int), ("lanes", C.c_int),
                ("rows", C.c_int), ("traceback", C.c_int), ("hb_cutoff", C.c_int),
                ("free_ends", C.c_int), ("soft_post", C.c_int)]


_lib = None


def lib():
    """Load (building first if needed) libnwgrad_b200.so."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB
    if not os.path.exists(path) or _build.stale():
        _build.build()
    L = C.CDLL(path)
    L.nwg_last_error.restype = C.c_char_p
    L.nwg_store_create.argtypes = [_u8p, _i64p, _u8p, _i64p, C.c_int64, C.c_int, _u16p, _u16p, C.c_int,
                                   C.POINTER(C.c_void_p)]
    L.nwg_store_destroy.argtypes = [C.c_void_p]
    L.nwg_params_set.argtypes = [C.c_void_p, _dp, _dp, C.c_int, C.c_int]
    L.nwg_run.argtypes = [C.c_void_p, C.POINTER(Job), C.c_void_p, _dp]
    L.nwg_scores.argtypes = [C.c_void_p, _dp]
    L.nwg_grads.argtypes = [C.c_void_p, _dp]
    L.nwg_reduce.argtypes = [C.c_void_p, _dp, _dp]
    L.nwg_guides.argtypes = [C.c_void_p, _i32p]
    L.nwg_set_guides.argtypes = [C.c_void_p, _i32p]
    L.nwg_resolve_guides.argtypes = [C.c_void_p, _dp, _dp, C.POINTER(Job), C.c_void_p]
    L.nwg_paths.argtypes = [C.c_void_p, _i64p, _u8p, C.c_int64, _i32p, _i32p]
    L.nwg_status.argtypes = [C.c_void_p, _i32p]
    L.nwg_last_timing.argtypes = [C.c_void_p, _dp, _i64p]
    L.nwg_set_memory.argtypes = [C.c_void_p, C.c_int64, C.c_int64]
    L.nwg_set_spin_limit.argtypes = [C.c_void_p, C.c_int]
    L.nwg_set_geometry.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int]
    L.nwg_set_graphs.argtypes = [C.c_void_p, C.c_int]
    L.nwg_set_geometry_costs.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _i32p, _i32p, _dp]
    L.nwg_graph_stats.argtypes = [C.c_void_p, _i64p, _i64p]
    for name in ("nwg_store_create", "nwg_store_destroy", "nwg_params_set", "nwg_run", "nwg_scores",
                 "nwg_grads", "nwg_reduce", "nwg_guides", "nwg_set_guides", "nwg_resolve_guides", "nwg_paths", "nwg_status",
                 "nwg_last_timing", "nwg_set_memory", "nwg_set_spin_limit", "nwg_set_geometry", "nwg_set_graphs", "nwg_graph_stats", "nwg_set_geometry_costs"):
        getattr(L, name).restype = C.c_int
    _lib = L
    return L


def check(rc: int):
    """Map a status to the reference's Python exceptions."""
    if rc == NWG_OK:
        return
    msg = lib().nwg_last_error().decode(errors="replace")
    if rc in (NWG_EINVAL, NWG_ERANGE):
        raise ValueError(msg)
    if rc == NWG_ESTATE:
        raise RuntimeError(msg)
    if rc == NWG_ENOMEM:
        raise MemoryError(msg)
    raise RuntimeError(f"CUDA error: {msg}")


def ptr(a, t):
    return None if a is None else a.ctypes.data_as(t)
