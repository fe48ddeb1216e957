"""The AdaptaHOP pipeline behind the drop-in boundary, as plain functions.

``configure`` performs the three parameter calls that the reference's driver
makes before each compute (init_adaptahop_130 / change_pos_1310 /
sync_fortran in src/compute_neiKDtree_mod.py:155-210, 738-747); ``run`` then
calls compute and returns the module outputs as numpy arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from compute_adaptahop import neikdtree


def configure(npart: int, box: float = 1.0, nvoisins: int = 32, nhop: int = 16, rho_threshold: float = 80.0,
              fudge: float = 4.0, fudgepsilon: float = 1e-5, alphap: float = 1.0, nmembthresh: int = 20,
              nlevelmax: int = 30, nusedpart: int | None = None):
    """Set parameters exactly as the reference's driver would for this box."""
    half = 0.5 * box
    # cosmology arguments are carried but unused by the finder (f90:591-641)
    neikdtree.sync_from_init_adaptahop(npart, nmembthresh, nmembthresh, 0.7, 0.7, 0.3, 0.3, 1.0, 1.0, 0.7, 70.0,
                                       box, box, box, box, box, half, half, half, 100.0, 1.0, [0.0, 0.0, 0.0])
    # change_pos_1310: epsilon = fudgepsilon * xlong / npart**(1/3)
    eps = fudgepsilon * box / npart ** (1.0 / 3.0)
    neikdtree.sync_from_change_pos(npart, npart if nusedpart is None else nusedpart, eps, fudgepsilon, box, box)
    neikdtree.sync_others(False, False, npart, 1, rho_threshold, 1.0 / npart, box, nhop, nvoisins, fudge, alphap,
                          "MSM", nlevelmax, False)
    return eps


def run(pos: np.ndarray, mass: np.ndarray) -> dict:
    """Run the full pipeline on host arrays pos (N,3) and mass (N,)."""
    pos = np.ascontiguousarray(pos, np.float64)
    neikdtree.compute_adaptahop(pos.T, mass)
    out = dict(density=neikdtree.density.copy(), liste_parts=neikdtree.liste_parts.copy(),
               nnodes=int(neikdtree.nnodes), real_table=np.ascontiguousarray(neikdtree.real_table.T),
               integer_table=np.ascontiguousarray(neikdtree.integer_table.T), timings=L.timings())
    o = L.AhopOutputs()
    L.check(L.lib().ahop_get_outputs(C.byref(o)), "get_outputs")
    out["ngroups"] = int(o.ngroups)
    return out


def run_stages(pos: np.ndarray, mass: np.ndarray, last_stage: int = 4, store_neighbours: int = 0) -> dict:
    """Run the pipeline up to a stage and return the stage views (1-based ids)."""
    pos = np.ascontiguousarray(pos, np.float64)
    mass = np.ascontiguousarray(mass, np.float64)
    n = mass.shape[0]
    lib = L.lib()
    L.check(lib.ahop_debug_set_store_neighbours(int(store_neighbours)), "set_store")
    L.check(lib.ahop_debug_compute_stages(pos.ctypes.data, mass.ctypes.data, n, int(last_stage)), "stages")
    out = {}
    dens = np.empty(n, np.float64)
    L.check(lib.ahop_debug_density(dens.ctypes.data), "density")
    out["density"] = dens
    if store_neighbours:
        nei = np.empty((n, store_neighbours), np.int32)
        L.check(lib.ahop_debug_neighbours(nei.ctypes.data, store_neighbours), "neighbours")
        out["neighbours"] = nei
    if last_stage >= 3:
        hop = np.empty(n, np.int32)
        grp = np.empty(n, np.int32)
        ng = C.c_int32()
        L.check(lib.ahop_debug_groups(hop.ctypes.data, grp.ctypes.data, C.byref(ng)), "groups")
        out.update(hop_target=hop, group_id=grp, ngroups=int(ng.value))
    if last_stage >= 4:
        nc = C.c_int32()
        L.check(lib.ahop_debug_saddles(C.byref(nc), None, None, None), "saddles")
        off = np.empty(out["ngroups"] + 1, np.int32)
        isad = np.empty(max(nc.value, 1), np.int32)
        rho = np.empty(max(nc.value, 1), np.float64)
        L.check(lib.ahop_debug_saddles(C.byref(nc), off.ctypes.data, isad.ctypes.data, rho.ctypes.data), "saddles")
        out.update(saddle_offsets=off, saddle_isad=isad[:nc.value].copy(), saddle_rho=rho[:nc.value].copy())
    L.check(lib.ahop_debug_set_store_neighbours(0), "set_store")
    return out
