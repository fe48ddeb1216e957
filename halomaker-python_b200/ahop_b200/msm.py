"""MSM halo/subhalo selection and member grouping through the C ABI.

After a finder compute, ``select()`` returns what select_with_MS_method_1319
(src/compute_neiKDtree_mod.py:260-464) and the grouping of NEI:107-119 leave
in the reference's shared arrays: structure id per particle
(whereIam_parts), the structure tree (mother/first_sister/first_daughter/
level) and the members grouped by structure.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L


class AhopStructs(C.Structure):
    _fields_ = [("nstruct", C.c_int32), ("nb_of_halos", C.c_int32), ("nb_of_subhalos", C.c_int32),
                ("ngroupruns", C.c_int32), ("nusedpart", C.c_int64), ("whereIam_parts", C.c_void_p),
                ("mother", C.c_void_p), ("first_sister", C.c_void_p), ("first_daughter", C.c_void_p),
                ("level", C.c_void_p), ("pids_groupsorted", C.c_void_p), ("run_ids", C.c_void_p),
                ("run_idxs", C.c_void_p), ("run_counts", C.c_void_p)]


def _arr(p, n):
    if n == 0:
        return np.empty(0, np.int32)
    return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_int32)), (n,)).copy()


def select(particle_views: bool = True) -> dict:
    """particle_views=False skips the per-particle host arrays (whereIam_parts,
    pids_groupsorted: None) -- for callers that gather members on the device."""
    lib = L.lib()
    lib.ahop_select_msm.argtypes = [C.POINTER(AhopStructs)]
    lib.ahop_msm_set_particle_views.argtypes = [C.c_int32]
    L.check(lib.ahop_msm_set_particle_views(int(bool(particle_views))), "msm_set_particle_views")
    o = AhopStructs()
    L.check(lib.ahop_select_msm(C.byref(o)), "select_msm")
    n, ns, nr = int(o.nusedpart), int(o.nstruct), int(o.ngroupruns)
    pv = lambda p: _arr(p, n) if particle_views else None
    return dict(nstruct=ns, nb_of_halos=int(o.nb_of_halos), nb_of_subhalos=int(o.nb_of_subhalos),
                whereIam_parts=pv(o.whereIam_parts), mother=_arr(o.mother, ns),
                first_sister=_arr(o.first_sister, ns), first_daughter=_arr(o.first_daughter, ns),
                level=_arr(o.level, ns), pids_groupsorted=pv(o.pids_groupsorted),
                run_ids=_arr(o.run_ids, nr), run_idxs=_arr(o.run_idxs, nr), run_counts=_arr(o.run_counts, nr))


def gather_device(d_pos, d_vel, d_mass, stream=None):
    """Members of every structure (id >= 1) gathered on the device in structure
    order, after ``select()``: returns (off int64[ns+1], ids int32[ns], pos,
    vel, mass, density) as torch CUDA tensors."""
    import torch
    lib = L.lib()
    lib.ahop_structure_members.argtypes = [C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
    lib.ahop_gather_members_device.argtypes = [C.c_void_p] * 10
    ns, nm = C.c_int32(), C.c_int64()
    L.check(lib.ahop_structure_members(C.byref(ns), C.byref(nm)), "structure_members")
    dev = d_pos.device
    off = torch.empty(ns.value + 1, dtype=torch.int64, device=dev)
    ids = torch.empty(max(ns.value, 1), dtype=torch.int32, device=dev)
    m = nm.value
    pos = torch.empty((max(m, 1), 3), dtype=torch.float64, device=dev)
    vel = torch.empty((max(m, 1), 3), dtype=torch.float64, device=dev) if d_vel is not None else None
    mass = torch.empty(max(m, 1), dtype=torch.float64, device=dev)
    dens = torch.empty(max(m, 1), dtype=torch.float64, device=dev)
    st = stream.cuda_stream if stream is not None else 0
    ptr = lambda t: t.data_ptr() if t is not None else None
    L.check(lib.ahop_gather_members_device(ptr(d_pos), ptr(d_vel), ptr(d_mass), ptr(off), ptr(ids), ptr(pos),
                                           ptr(vel), ptr(mass), ptr(dens), st), "gather_members_device")
    return off, ids[:ns.value], pos[:m], (vel[:m] if vel is not None else None), mass[:m], dens[:m]


def gather_index_device(nmembers, device, stream=None):
    """Particle index (0-based, caller's order) of every member gathered by
    gather_device, in the same order, as an int32 CUDA tensor."""
    import torch
    lib = L.lib()
    lib.ahop_gather_member_index_device.argtypes = [C.c_void_p, C.c_void_p]
    idx = torch.empty(max(int(nmembers), 1), dtype=torch.int32, device=device)
    st = stream.cuda_stream if stream is not None else 0
    L.check(lib.ahop_gather_member_index_device(idx.data_ptr(), st), "gather_member_index_device")
    return idx[:int(nmembers)]
