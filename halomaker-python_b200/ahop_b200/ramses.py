"""RAMSES particle files read through the device decoder (ahop_ramses_*).

The reference reads particles with read_ramses_new_101 /
_read_ramses_new_1010 (src/input_output.py:763-989, 624-760) into the shared
arrays pos_10, vel_10, mass_10 (and source_pid_10 for a single family); this
module produces the same arrays as torch CUDA tensors, ready for the finder's
device entry point.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib as L

FAMILIES = {"all": 0, "dm": 1, "star": 2}


class AhopRamsesParams(C.Structure):
    _fields_ = [("version", C.c_int32), ("family", C.c_int32), ("scale_l", C.c_double), ("scale_t", C.c_double)]


class AhopRamsesCounts(C.Structure):
    _fields_ = [("total", C.c_int64), ("ndm", C.c_int64), ("nstar", C.c_int64), ("nselected", C.c_int64),
                ("nfiles", C.c_int32), ("ndim", C.c_int32)]


def read_info(path: str) -> dict:
    """scale_l / scale_d / scale_t / H0 from a RAMSES info file, as
    _read_ramses_info_params reads them (input_output.py:124-142)."""
    params = {}
    conv = lambda v: np.float64(str(v).replace("D", "E").replace("d", "e"))
    with open(path) as f:
        for line in f:
            line = line.strip()
            if not line or line.startswith("#") or "=" not in line:
                continue
            name, value = (t.strip() for t in line.split("=", 1))
            if "!" in value:
                value = value.split("!")[0].strip()
            if name in ("unit_l", "scale_l"):
                params["scale_l"] = conv(value)
            elif name in ("unit_d", "scale_d"):
                params["scale_d"] = conv(value)
            elif name in ("unit_t", "scale_t"):
                params["scale_t"] = conv(value)
            elif name == "H0":
                params["H0"] = conv(value)
    return params


def part_files(repository: str) -> list:
    """part_<nchar>.out<icpu> for icpu = 1..ncpu of an output_<nchar> directory
    (ncpu from the first file's header, as the reference reads it)."""
    ipos = repository.find("output_")
    if ipos < 0:
        raise ValueError("repository must be an output_NNNNN directory")
    nchar = repository[ipos + 7:ipos + 12]
    first = os.path.join(repository, f"part_{nchar}.out00001")
    with open(first, "rb") as f:
        n = np.frombuffer(f.read(4), np.uint32)[0]
        ncpu = int(np.frombuffer(f.read(n), np.int32)[0])
    return [os.path.join(repository, f"part_{nchar}.out{i:05d}") for i in range(1, ncpu + 1)]


def read_parts(files, version: int = 3, family: str = "all", scale_l: float = 1.0, scale_t: float = 1.0,
               stream=None) -> dict:
    """files: an output_NNNNN directory or the part file paths in cpu order.

    Returns pos (n,3), vel (n,3), mass (n,) [and source_pid (n,) for a single
    family] as torch CUDA tensors plus the family counts."""
    import torch
    if isinstance(files, str):
        files = part_files(files)
    lib = L.lib()
    lib.ahop_ramses_open.argtypes = [C.c_void_p, C.c_int32, C.POINTER(AhopRamsesParams), C.POINTER(AhopRamsesCounts)]
    lib.ahop_ramses_decode_device.argtypes = [C.c_void_p] * 5
    arr = (C.c_char_p * len(files))(*[os.fsencode(p) for p in files])
    prm = AhopRamsesParams(int(version), FAMILIES[family], float(scale_l), float(scale_t))
    cnt = AhopRamsesCounts()
    L.check(lib.ahop_ramses_open(arr, len(files), C.byref(prm), C.byref(cnt)), "ramses_open")
    n = int(cnt.nselected)
    dev = torch.device("cuda")
    pos = torch.empty((n, 3), dtype=torch.float64, device=dev)
    vel = torch.empty((n, 3), dtype=torch.float64, device=dev)
    mass = torch.empty(n, dtype=torch.float64, device=dev)
    spid = torch.empty(n, dtype=torch.int64, device=dev) if family != "all" else None
    st = stream.cuda_stream if stream is not None else torch.cuda.current_stream().cuda_stream
    try:
        L.check(lib.ahop_ramses_decode_device(pos.data_ptr(), vel.data_ptr(), mass.data_ptr(),
                                              spid.data_ptr() if spid is not None else None, st), "ramses_decode")
    finally:
        lib.ahop_ramses_close()
    out = dict(pos=pos, vel=vel, mass=mass, ndm=int(cnt.ndm), nstar=int(cnt.nstar), nselected=n,
               total=int(cnt.total))
    if spid is not None:
        out["source_pid"] = spid
    return out
