"""Batched per-halo properties through the C ABI (ahop_halo_props*).

Replaces the per-halo property chain of the reference
(_compute_halo_props, src/compute_halo_props.py:270-301) for the fields it
lists: mass with its dark-matter / star split, centre (densest member, the
member closest to the centre of mass with cdm, or the shrinking sphere),
bulk velocity, sigma (all, dark matter, stars), angular momentum, r, inertia
tensor and principal axes, E_kin (with Hubble flow), the direct-sum E_pot in
FP64 and FP32-compensated forms, and spin.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

FIELDS = ["m", "px", "py", "pz", "vx", "vy", "vz", "Lx", "Ly", "Lz", "r", "Ixx", "Ixy", "Ixz", "Iyy", "Iyz",
          "Izz", "ek", "ep64", "ep32c", "sigma", "sha", "shb", "shc", "spin64", "spin32c", "icenter",
          "ndm", "nstar", "mdm", "m*", "mcontam", "sigma_dm", "sigma*"]
NF = len(FIELDS)


class AhopHaloParams(C.Structure):
    _fields_ = [("Lbox", C.c_double), ("Hub_pt", C.c_double), ("gravconst", C.c_double),
                ("periodic", C.c_int32), ("epot", C.c_int32), ("sc", C.c_int32), ("pad", C.c_int32),
                ("dcell_min", C.c_double), ("eps_sc", C.c_double), ("cdm", C.c_int32), ("pad2", C.c_int32),
                ("ndm", C.c_int64), ("massp", C.c_double), ("index", C.c_void_p)]


class AhopHaloTimings(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("moments", "epot64", "epot32c", "finalize", "total")] + [
        ("pairs", C.c_double), ("items", C.c_int32), ("kernel_launches", C.c_int32), ("tune_ms", C.c_float),
        ("graph_replays", C.c_int32)]


BUCKETS = 5  # halo-size buckets of the FP32 pair kernel's tile shape: n < 512, 4096, 32768, 262144, larger


_bound = False


def _lib():
    global _bound
    lib = L.lib()
    if not _bound:
        lib.ahop_halo_props.argtypes = [C.POINTER(AhopHaloParams), C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ahop_halo_props_device.argtypes = [C.POINTER(AhopHaloParams), C.c_void_p, C.c_int64, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        lib.ahop_halo_get_timings.argtypes = [C.POINTER(AhopHaloTimings)]
        lib.ahop_halo_get_tiles.argtypes = [C.c_void_p, C.c_void_p]
        lib.ahop_halo_set_tiles.argtypes = [C.c_void_p]
        lib.ahop_halo_set_graph.argtypes = [C.c_int32]
        _bound = True
    return lib


def params(Lbox, Hub_pt, gravconst=430.1, periodic=True, epot=3, sc=None, cdm=False, ndm=None, massp=0.0,
           index=None):
    """sc: None (centre = densest member) or (dcell_min, eps_SC) for the
    shrinking-sphere centre of refine_centers_1b.  cdm: centre = member
    closest to the centre of mass (H.cdm).  index: the members' particle
    indices (a pointer in the memory of the call's other arrays, or None:
    every member is dark matter); members with index < ndm are dark matter
    (H.ndm), those heavier than massp * 1.00001 count as contamination."""
    on = sc is not None
    return AhopHaloParams(float(Lbox), float(Hub_pt), float(gravconst), int(bool(periodic)), int(epot), int(on), 0,
                          float(sc[0]) if on else 0.0, float(sc[1]) if on else 0.0, int(bool(cdm)), 0,
                          int(ndm if ndm is not None else 2 ** 62), float(massp), index)


def compute(off, pos, vel, mass, dens, Lbox, Hub_pt, gravconst=430.1, periodic=True, epot=3, sc=None, cdm=False,
            index=None, ndm=None, massp=0.0) -> dict:
    """Host arrays in, dict of per-halo arrays out (FIELDS).  index: the
    members' particle indices (int32, the reference's indexps), members with
    index < ndm being dark matter; None: every member is dark matter."""
    off = np.ascontiguousarray(off, np.int64)
    nh = len(off) - 1
    pos = np.ascontiguousarray(pos, np.float64)
    vel = np.ascontiguousarray(vel, np.float64)
    mass = np.ascontiguousarray(mass, np.float64)
    dens = np.ascontiguousarray(dens, np.float64)
    out = np.zeros((max(nh, 1), NF))
    idx = None if index is None else np.ascontiguousarray(index, np.int32)
    p = params(Lbox, Hub_pt, gravconst, periodic, epot, sc, cdm, ndm, massp,
               None if idx is None else idx.ctypes.data)
    L.check(_lib().ahop_halo_props(C.byref(p), off.ctypes.data, nh, pos.ctypes.data, vel.ctypes.data,
                                   mass.ctypes.data, dens.ctypes.data, out.ctypes.data), "halo_props")
    return {f: out[:nh, k].copy() for k, f in enumerate(FIELDS)}


def compute_device(d_off, d_pos, d_vel, d_mass, d_dens, d_out, Lbox, Hub_pt, gravconst=430.1, periodic=True,
                   epot=3, stream=None, sc=None, cdm=False, d_index=None, ndm=None, massp=0.0):
    """torch CUDA tensors in; fills d_out (nhalo, NF) in place.  d_index: the
    members' particle indices (int32 tensor) or None."""
    p = params(Lbox, Hub_pt, gravconst, periodic, epot, sc, cdm, ndm, massp,
               None if d_index is None else d_index.data_ptr())
    nh = d_off.numel() - 1
    st = C.c_void_p(stream.cuda_stream if stream is not None else 0)
    L.check(_lib().ahop_halo_props_device(C.byref(p), d_off.data_ptr(), nh, d_pos.data_ptr(), d_vel.data_ptr(),
                                          d_mass.data_ptr(), d_dens.data_ptr(), d_out.data_ptr(), st),
            "halo_props_device")


def compute_device_noalloc(d_off, d_pos, d_vel, d_mass, d_dens, d_out, Lbox, Hub_pt, gravconst=430.1,
                           periodic=True, epot=3, stream=None):
    """Same as compute_device, through the allocation-free entry point
    (ahop_halo_props_noalloc): no device memory is allocated by the call.
    The default stream is torch's current stream.  The call blocks the host
    twice and refuses a capturing stream; next to another thread's capture
    pass a non-blocking stream (the legacy default stream would join it)."""
    lib = _lib()
    lib.ahop_halo_props_noalloc.argtypes = [C.POINTER(AhopHaloParams), C.c_void_p, C.c_int64, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    p = params(Lbox, Hub_pt, gravconst, periodic, epot)
    nh = d_off.numel() - 1
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    st = C.c_void_p(stream.cuda_stream)
    L.check(lib.ahop_halo_props_noalloc(C.byref(p), d_off.data_ptr(), nh, d_pos.data_ptr(), d_vel.data_ptr(),
                                        d_mass.data_ptr(), d_dens.data_ptr(), d_out.data_ptr(), st),
            "halo_props_noalloc")


def timings() -> dict:
    t = AhopHaloTimings()
    L.check(_lib().ahop_halo_get_timings(C.byref(t)), "halo_get_timings")
    return {n: getattr(t, n) for n, _ in AhopHaloTimings._fields_}


def tiles() -> dict:
    """Rows per work item of the FP32-compensated pair kernel per halo-size
    bucket (0 = not tuned yet) and the autotuner's times (ms) per shape."""
    rows = np.zeros(BUCKETS, np.int32)
    ms = np.zeros(BUCKETS * 3, np.float32)
    L.check(_lib().ahop_halo_get_tiles(rows.ctypes.data, ms.ctypes.data), "halo_get_tiles")
    return {"rows": rows.tolist(), "tune_ms": ms.reshape(BUCKETS, 3).tolist()}


def set_tiles(rows=None) -> None:
    """Pin rows per item (128, 256 or 512; 0 = autotune) per bucket; None
    forgets every pin and every tuned shape."""
    if rows is None:
        L.check(_lib().ahop_halo_set_tiles(None), "halo_set_tiles")
        return
    r = np.ascontiguousarray(rows, np.int32)
    if r.shape != (BUCKETS,):
        raise ValueError(f"rows must have {BUCKETS} entries")
    L.check(_lib().ahop_halo_set_tiles(r.ctypes.data), "halo_set_tiles")


def set_graph(on: bool) -> None:
    """Capture and replay the launch sequence as a CUDA graph (default on)."""
    L.check(_lib().ahop_halo_set_graph(int(bool(on))), "halo_set_graph")


# ---------------------------------------------------------------- virial step
VIR_FIELDS = ["rvir", "mvir", "cvel", "tvir", "rho_0", "r_c", "ep", "et", "amax", "bmax", "cmax"]
NV = len(VIR_FIELDS)


class AhopVirialParams(C.Structure):
    _fields_ = [("Lbox", C.c_double), ("Hub_pt", C.c_double), ("gravconst", C.c_double),
                ("vir_overdens", C.c_double), ("rho_mean", C.c_double), ("periodic", C.c_int32),
                ("nshell", C.c_int32), ("direct_limit", C.c_int32), ("ep_field", C.c_int32)]


def virial_params(Lbox, Hub_pt, gravconst, vir_overdens, rho_mean, periodic=True, nshell=1000, direct_limit=1000,
                  ep="ep64"):
    return AhopVirialParams(float(Lbox), float(Hub_pt), float(gravconst), float(vir_overdens), float(rho_mean),
                            int(bool(periodic)), int(nshell), int(direct_limit), FIELDS.index(ep))


def virial(off, pos, vel, mass, props, Lbox, Hub_pt, gravconst=430.1, vir_overdens=178.0, rho_mean=1.0,
           periodic=True, nshell=1000, direct_limit=1000, ep="ep64") -> dict:
    """det_vir_1b for every halo (ahop_halo_virial).  props: the dict returned
    by compute() for the same halos.  Returns a dict of per-halo arrays
    (VIR_FIELDS); ep/et are the reference's final energies."""
    lib = _lib()
    lib.ahop_halo_virial.argtypes = [C.POINTER(AhopVirialParams), C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                     C.c_void_p, C.c_void_p, C.c_void_p]
    off = np.ascontiguousarray(off, np.int64)
    nh = len(off) - 1
    pos = np.ascontiguousarray(pos, np.float64)
    vel = np.ascontiguousarray(vel, np.float64)
    mass = np.ascontiguousarray(mass, np.float64)
    rows = np.ascontiguousarray(np.stack([np.asarray(props[f], np.float64) for f in FIELDS], 1)) if nh else \
        np.zeros((1, NF))
    out = np.zeros((max(nh, 1), NV))
    p = virial_params(Lbox, Hub_pt, gravconst, vir_overdens, rho_mean, periodic, nshell, direct_limit, ep)
    L.check(lib.ahop_halo_virial(C.byref(p), off.ctypes.data, nh, pos.ctypes.data, vel.ctypes.data,
                                 mass.ctypes.data, rows.ctypes.data, out.ctypes.data), "halo_virial")
    return {f: out[:nh, k].copy() for k, f in enumerate(VIR_FIELDS)}


def virial_device(d_off, d_pos, d_vel, d_mass, d_props, d_out, Lbox, Hub_pt, gravconst=430.1, vir_overdens=178.0,
                  rho_mean=1.0, periodic=True, nshell=1000, direct_limit=1000, ep="ep64", stream=None):
    """torch CUDA tensors in (d_props: the (nhalo, NF) output of compute_device);
    fills d_out (nhalo, NV) in place."""
    lib = _lib()
    lib.ahop_halo_virial_device.argtypes = [C.POINTER(AhopVirialParams), C.c_void_p, C.c_int64, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    p = virial_params(Lbox, Hub_pt, gravconst, vir_overdens, rho_mean, periodic, nshell, direct_limit, ep)
    nh = d_off.numel() - 1
    st = C.c_void_p(stream.cuda_stream if stream is not None else 0)
    L.check(lib.ahop_halo_virial_device(C.byref(p), d_off.data_ptr(), nh, d_pos.data_ptr(), d_vel.data_ptr(),
                                        d_mass.data_ptr(), d_props.data_ptr(), d_out.data_ptr(), st),
            "halo_virial_device")


def virial_last_ms() -> float:
    lib = _lib()
    lib.ahop_halo_virial_last_ms.restype = C.c_float
    return float(lib.ahop_halo_virial_last_ms())
