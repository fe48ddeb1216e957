"""ctypes binding of libahop_b200.so (C ABI in include/ahop_b200.h).

The library is the only implementation: if it is missing or fails to load,
every call raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libahop_b200.so")

AHOP_ERRORS = {1: "EINVAL", 2: "ECUDA", 3: "ENOMEM", 4: "ESTATE", 5: "EINVARIANT", 6: "ELIMIT", 7: "EDATA", 8: "EIO"}


class AhopInit(C.Structure):
    _fields_ = [("npart", C.c_int64), ("nmembthresh", C.c_int32), ("nMembers", C.c_int32)] + [
        (n, C.c_double) for n in ("omegaL", "omega_lambda_f", "omega0", "omega_f", "aexp_max", "af", "hubble",
                                  "H_f", "boxsize2", "Lf", "xlong", "ylong", "zlong", "xlongs2", "ylongs2",
                                  "zlongs2", "Hub_pt", "aexp")] + [("pos_shift", C.c_double * 3)]


class AhopOthers(C.Structure):
    _fields_ = [("verbose", C.c_int32), ("megaverbose", C.c_int32), ("npart", C.c_int32), ("nbPes", C.c_int32),
                ("rho_threshold", C.c_double), ("massp", C.c_double), ("boxsize", C.c_double),
                ("nhop", C.c_int32), ("nvoisins", C.c_int32), ("fudge", C.c_double), ("alphap", C.c_double),
                ("method", C.c_char * 8), ("nlevelmax", C.c_int32), ("optimize_nodes", C.c_int32)]


class AhopOutputs(C.Structure):
    _fields_ = [("npart", C.c_int64), ("nusedpart", C.c_int64), ("nnodes", C.c_int32), ("ngroups", C.c_int32),
                ("liste_parts", C.c_void_p), ("density", C.c_void_p), ("real_table", C.c_void_p),
                ("integer_table", C.c_void_p)]


class AhopTimings(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("upload", "tree", "knn_density", "hop_groups", "saddles", "nodes",
                                         "membership", "download", "total", "knn_kernel", "nodes_prep",
                                         "nodes_root", "nodes_waves", "nodes_order")] + [
        (n, C.c_int32) for n in ("kernel_launches", "cub_calls", "tree_waves", "hop_passes")]


class AhopError(RuntimeError):
    pass


_lib = None
_lock = threading.Lock()

_SIGS = {
    "ahop_sync_from_init_adaptahop": [C.POINTER(AhopInit)],
    "ahop_sync_from_change_pos": [C.c_int64, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double],
    "ahop_sync_others": [C.POINTER(AhopOthers)],
    "ahop_compute_adaptahop": [C.c_void_p, C.c_void_p, C.c_int64],
    "ahop_compute_adaptahop_device": [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p],
    "ahop_get_outputs": [C.POINTER(AhopOutputs)],
    "ahop_get_device_outputs": [C.POINTER(AhopOutputs)],
    "ahop_get_timings": [C.POINTER(AhopTimings)],
    "ahop_close": [],
    "ahop_release_device_memory": [],
    "ahop_debug_neighbours": [C.c_void_p, C.c_int32],
    "ahop_debug_density": [C.c_void_p],
    "ahop_debug_groups": [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32)],
    "ahop_debug_saddles": [C.POINTER(C.c_int32), C.c_void_p, C.c_void_p, C.c_void_p],
    "ahop_debug_compute_stages": [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32],
    "ahop_debug_set_store_neighbours": [C.c_int32],
    "ahop_debug_tree_stats": [C.c_void_p, C.c_int32],
}


def lib():
    """Load the CUDA library (raises if it is missing: there is no fallback)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise AhopError(f"{LIB_PATH} is missing: build it with ahop_b200.build.build()")
            L = C.CDLL(LIB_PATH)
            L.ahop_last_error.restype = C.c_char_p
            for name, args in _SIGS.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = C.c_int
            _lib = L
    return _lib


def check(rc: int, what: str = ""):
    if rc != 0:
        msg = lib().ahop_last_error().decode(errors="replace")
        raise AhopError(f"{what or 'ahop'} failed [{AHOP_ERRORS.get(rc, rc)}]: {msg}")


def ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def timings() -> dict:
    t = AhopTimings()
    check(lib().ahop_get_timings(C.byref(t)), "ahop_get_timings")
    return {n: (float(getattr(t, n)) if ty is C.c_float else int(getattr(t, n))) for n, ty in AhopTimings._fields_}
