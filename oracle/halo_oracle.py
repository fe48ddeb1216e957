"""CPU oracle for the batched halo properties -- TEST INFRASTRUCTURE ONLY.

O(n) fields restate the reference's NumPy reductions (src/compute_halo_props.py:
det_mass_17 754-780, det_center_18 901-966, compute_ang_mom_19 783-824,
r_halos_1a 828-851, det_inertial_tensor_1b20/det_main_axis_1b2 1932-1967,
det_halo_energies_1b3 1430-1444, compute_spin_parameter_1c 1599-1602);
the O(n^2) potential comes from halo_props_oracle.cpp (FP64 direct sum).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None

FIELDS = ["m", "px", "py", "pz", "vx", "vy", "vz", "Lx", "Ly", "Lz", "r", "Ixx", "Ixy", "Ixz", "Iyy", "Iyz",
          "Izz", "ek", "ep64", "ep32c", "sigma", "sha", "shb", "shc", "spin64", "spin32c", "icenter"]


def lib():
    global _lib
    if _lib is None:
        so = os.path.join(_HERE, "_build", "libhalo_oracle.so")
        src = os.path.join(_HERE, "halo_props_oracle.cpp")
        if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
            subprocess.check_call(["make", "-s", "-C", _HERE, os.path.join("_build", "libhalo_oracle.so")])
        _lib = C.CDLL(so)
        _lib.halo_oracle_epot.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_double, C.c_int,
                                          C.c_int, C.c_void_p]
    return _lib


def epot_sums(off, pos, mass, L, periodic=True, nthreads=None):
    off = np.ascontiguousarray(off, np.int64)
    pos = np.ascontiguousarray(pos, np.float64)
    mass = np.ascontiguousarray(mass, np.float64)
    out = np.zeros(len(off) - 1)
    lib().halo_oracle_epot(off.ctypes.data, len(off) - 1, pos.ctypes.data, mass.ctypes.data, float(L),
                           int(bool(periodic)), int(nthreads or os.cpu_count()), out.ctypes.data)
    return out


def _wrap(d, L):
    d = d.copy()
    d[d > L / 2] -= L
    d[d < -L / 2] += L
    return d


def props(off, pos, vel, mass, dens, L, hub, G=430.1, periodic=True, epot=True, nthreads=None):
    """Per-halo fields as a dict of arrays (names as in FIELDS, ep = FP64 pair sum)."""
    nh = len(off) - 1
    res = {f: np.zeros(nh) for f in FIELDS}
    for h in range(nh):
        a, b = off[h], off[h + 1]
        p, v, m, d = pos[a:b], vel[a:b], mass[a:b], dens[a:b]
        mt = np.sum(m)
        ic = int(np.argmax(d))
        c = p[ic]
        vb = np.array([np.sum(m * v[:, 0]), np.sum(m * v[:, 1]), np.sum(m * v[:, 2])]) / mt
        dr = np.stack([_wrap(p[:, k] - c[k], L) if periodic else p[:, k] - c[k] for k in range(3)], 1)
        u = v - vb
        pv = m[:, None] * u
        Lv = np.array([np.sum(dr[:, 1] * pv[:, 2] - dr[:, 2] * pv[:, 1]), np.sum(dr[:, 2] * pv[:, 0] - dr[:, 0] * pv[:, 2]),
                       np.sum(dr[:, 0] * pv[:, 1] - dr[:, 1] * pv[:, 0])])
        I = np.array([[np.sum(m * dr[:, i] * dr[:, j]) for j in range(3)] for i in range(3)])
        ev = np.linalg.eigvalsh(I)
        t = u + dr * hub
        res["m"][h] = mt
        res["px"][h], res["py"][h], res["pz"][h] = c
        res["vx"][h], res["vy"][h], res["vz"][h] = vb
        res["Lx"][h], res["Ly"][h], res["Lz"][h] = Lv
        res["r"][h] = np.sqrt(np.max(np.sum(dr * dr, 1)))
        for k, f in enumerate(["Ixx", "Ixy", "Ixz", "Iyy", "Iyz", "Izz"]):
            res[f][h] = I[[0, 0, 0, 1, 1, 2][k], [0, 1, 2, 1, 2, 2][k]]
        res["ek"][h] = 0.5 * np.sum(m * np.sum(t * t, 1))
        res["sigma"][h] = np.sqrt(np.sum(m * np.sum(u * u, 1)) / mt)
        res["sha"][h], res["shb"][h], res["shc"][h] = np.sqrt(ev / mt)
        res["icenter"][h] = ic
    if epot:
        s = epot_sums(off, pos, mass, L, periodic, nthreads)
        res["ep64"] = -G * s
        hl = np.sqrt(res["Lx"] ** 2 + res["Ly"] ** 2 + res["Lz"] ** 2)
        res["spin64"] = hl * np.sqrt(np.abs(res["ek"] + res["ep64"])) / res["m"] ** 2.5 / G
    return res
