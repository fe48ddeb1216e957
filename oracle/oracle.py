"""ctypes front-end of the CPU oracle — TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg may
import this module.  It restates the reference's finder
(fortran/compute_adaptahop.f90) on the CPU and is the checker for the CUDA
path; the product library never calls it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")
_lib = None


class OracleParams(C.Structure):
    _fields_ = [("npart", C.c_int64), ("nvoisins", C.c_int32), ("nhop", C.c_int32),
                ("nlevelmax", C.c_int32), ("nmembthresh", C.c_int32), ("nthreads", C.c_int32),
                ("rho_threshold", C.c_double), ("fudge", C.c_double), ("alphap", C.c_double),
                ("epsilon", C.c_double), ("xlong", C.c_double), ("ylong", C.c_double),
                ("zlong", C.c_double), ("xlongs2", C.c_double), ("ylongs2", C.c_double),
                ("zlongs2", C.c_double)]


class OracleResult(C.Structure):
    _fields_ = [("ngroups", C.c_int32), ("nnodes", C.c_int32), ("ncells", C.c_int32),
                ("pad", C.c_int32), ("stage_seconds", C.c_double * 4)]


class OracleCapture(C.Structure):
    _fields_ = [("neighbours", C.c_void_p), ("neighbours_k", C.c_int32), ("hop_target", C.c_void_p),
                ("group_id", C.c_void_p), ("keep_saddles", C.c_int32)]


def build(force: bool = False) -> str:
    so = os.path.join(_BUILD, "libahop_oracle.so")
    if force or not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(
            os.path.join(_HERE, "ahop_oracle.cpp")):
        subprocess.check_call(["make", "-s", "-C", _HERE, os.path.join("_build", "libahop_oracle.so")])
    return so


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        _lib.oracle_last_error.restype = C.c_char_p
        _lib.oracle_adaptahop.argtypes = [C.POINTER(OracleParams), C.c_void_p, C.c_void_p,
                                          C.POINTER(OracleResult), C.POINTER(OracleCapture)]
        _lib.oracle_copy_outputs.argtypes = [C.c_void_p] * 4
        _lib.oracle_saddles.argtypes = [C.POINTER(C.c_int32), C.c_void_p, C.c_void_p, C.c_void_p]
    return _lib


def default_params(npart, box=1.0, nvoisins=32, nhop=16, rho_threshold=80.0, fudge=4.0,
                   fudgepsilon=1e-5, alphap=1.0, nmembthresh=20, nlevelmax=30, nthreads=None):
    # epsilon as change_pos_1310 computes it (src/compute_neiKDtree_mod.py:203)
    eps = fudgepsilon * box / npart ** (1.0 / 3.0)
    return dict(npart=npart, nvoisins=nvoisins, nhop=nhop, nlevelmax=nlevelmax, nmembthresh=nmembthresh,
                nthreads=nthreads or os.cpu_count(), rho_threshold=rho_threshold, fudge=fudge,
                alphap=alphap, epsilon=eps, xlong=box, ylong=box, zlong=box,
                xlongs2=box * 0.5, ylongs2=box * 0.5, zlongs2=box * 0.5)


def run(pos, mass, params: dict, capture_neighbours: int = 0, capture_hop: bool = False,
        capture_saddles: bool = False):
    """Run the oracle on pos (N,3) / mass (N,).  Returns a dict of outputs."""
    L = lib()
    pos = np.ascontiguousarray(pos, np.float64)
    mass = np.ascontiguousarray(mass, np.float64)
    n = mass.shape[0]
    p = OracleParams(**params)
    res = OracleResult()
    cap = OracleCapture()
    out = {}
    if capture_neighbours:
        nei = np.empty((n, capture_neighbours), np.int32)
        cap.neighbours = nei.ctypes.data
        cap.neighbours_k = capture_neighbours
        out["neighbours"] = nei
    if capture_hop:
        hop = np.empty(n, np.int32)
        grp = np.empty(n, np.int32)
        cap.hop_target = hop.ctypes.data
        cap.group_id = grp.ctypes.data
        out["hop_target"] = hop
        out["group_id"] = grp
    cap.keep_saddles = 1 if capture_saddles else 0
    rc = L.oracle_adaptahop(C.byref(p), pos.ctypes.data, mass.ctypes.data, C.byref(res), C.byref(cap))
    if rc != 0:
        raise RuntimeError(f"oracle failed ({rc}): {L.oracle_last_error().decode()}")
    nn = res.nnodes
    dens = np.empty(n, np.float64)
    lp = np.empty(n, np.int32)
    rt = np.empty((max(nn, 1), 8), np.float64)
    it = np.empty((max(nn, 1), 6), np.int32)
    L.oracle_copy_outputs(dens.ctypes.data, lp.ctypes.data, rt.ctypes.data, it.ctypes.data)
    out.update(density=dens, liste_parts=lp, real_table=rt[:nn].copy(), integer_table=it[:nn].copy(),
               nnodes=nn, ngroups=res.ngroups, ncells=res.ncells,
               stage_seconds=list(res.stage_seconds))
    if capture_saddles:
        ng = res.ngroups
        nconn = C.c_int32()
        L.oracle_saddles(C.byref(nconn), None, None, None)
        off = np.empty(ng + 1, np.int32)
        isad = np.empty(max(nconn.value, 1), np.int32)
        rho = np.empty(max(nconn.value, 1), np.float64)
        L.oracle_saddles(C.byref(nconn), off.ctypes.data, isad.ctypes.data, rho.ctypes.data)
        out["saddle_offsets"] = off
        out["saddle_isad"] = isad[:nconn.value].copy()
        out["saddle_rho"] = rho[:nconn.value].copy()
    L.oracle_release()
    return out
