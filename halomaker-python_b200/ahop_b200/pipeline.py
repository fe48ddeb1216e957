"""One snapshot through the GPU: finder, MSM selection, member gather and the
batched halo properties.

This is the reference's snapshot step (new_step_1, src/compute_halo_props.py:304):
make_halos_13 runs compute_adaptahop_131 (src/compute_neiKDtree_mod.py:39-124:
the finder, select_with_MS_method_1319 and the member grouping), then the
per-structure loop (CHP:487-534) gathers each structure's members through
pids0_groupsorted / whereIam_idxs and runs _compute_halo_props on them.  Here
the particle arrays go to the device once; the finder, the selection, the
gather and the property launch all read device memory, and only the
selection's host views and the property rows come back.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import _lib as L
from . import finder, halo_props, msm, ramses


def run_snapshot(pos: np.ndarray, vel: np.ndarray, mass: np.ndarray, box: float = 1.0, hub: float = 70.0,
                 gravconst: float = 430.1, epot: int = 2, finder_params: dict | None = None,
                 particle_views: bool = False) -> dict:
    """Host arrays pos (N,3), vel (N,3), mass (N,) in box units ([-box/2, box/2)).

    Returns the structure selection (ids, tree arrays; the per-particle arrays
    whereIam_parts / pids_groupsorted only with particle_views), one property
    row per structure with members (halo_props.FIELDS, structure order =
    ascending id) and per-stage times in ms (device stages by CUDA events, the
    rest by the host clock around synchronised steps)."""
    import torch
    n = int(mass.shape[0])
    finder.configure(n, box=box, **(finder_params or {}))
    dev = torch.device("cuda")
    times = {}
    t0 = time.perf_counter()
    h_pos = torch.from_numpy(np.ascontiguousarray(pos, np.float64)).pin_memory()
    h_vel = torch.from_numpy(np.ascontiguousarray(vel, np.float64)).pin_memory()
    h_mass = torch.from_numpy(np.ascontiguousarray(mass, np.float64)).pin_memory()
    times["pin"] = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    d_pos = h_pos.to(dev, non_blocking=True)
    d_vel = h_vel.to(dev, non_blocking=True)
    d_mass = h_mass.to(dev, non_blocking=True)
    torch.cuda.synchronize()
    times["h2d"] = (time.perf_counter() - t0) * 1e3
    return _run_device(d_pos, d_vel, d_mass, box, hub, gravconst, epot, particle_views, times)


def _run_device(d_pos, d_vel, d_mass, box, hub, gravconst, epot, particle_views, times):
    """Finder, selection, member gather and properties on device arrays."""
    import torch
    n = int(d_mass.shape[0])
    dev = d_pos.device
    st = torch.cuda.current_stream()
    lib = L.lib()
    t0 = time.perf_counter()
    L.check(lib.ahop_compute_adaptahop_device(d_pos.data_ptr(), d_mass.data_ptr(), n, C.c_void_p(st.cuda_stream)),
            "compute_adaptahop_device")
    torch.cuda.synchronize()
    times["finder"] = (time.perf_counter() - t0) * 1e3
    times["finder_stages"] = L.timings()
    t0 = time.perf_counter()
    sel = msm.select(particle_views=particle_views)
    times["msm"] = (time.perf_counter() - t0) * 1e3
    t0 = time.perf_counter()
    off, ids, gpos, gvel, gmass, gdens = msm.gather_device(d_pos, d_vel, d_mass, stream=st)
    torch.cuda.synchronize()
    times["gather"] = (time.perf_counter() - t0) * 1e3
    ns = int(ids.numel())
    out = torch.empty((max(ns, 1), halo_props.NF), dtype=torch.float64, device=dev)
    t0 = time.perf_counter()
    if ns:
        halo_props.compute_device(off, gpos, gvel, gmass, gdens, out, box, hub, gravconst, True, epot, stream=st)
    torch.cuda.synchronize()
    times["props"] = (time.perf_counter() - t0) * 1e3
    times["props_stages"] = halo_props.timings() if ns else {}
    t0 = time.perf_counter()
    rows = out[:ns].cpu().numpy()
    ids_h = ids.cpu().numpy()
    off_h = off.cpu().numpy()
    times["d2h"] = (time.perf_counter() - t0) * 1e3
    return dict(sel, ids=ids_h, offsets=off_h, props=rows, members=int(off_h[-1]) if ns else 0, timings=times)


def run_snapshot_files(repository, version: int = 3, family: str = "all", scale_l: float = 1.0,
                       scale_t: float = 1.0, box: float = 1.0, hub: float = 70.0, gravconst: float = 430.1,
                       epot: int = 2, finder_params: dict | None = None, particle_views: bool = False) -> dict:
    """The same snapshot step starting from RAMSES part files (an
    output_NNNNN directory or the file paths): read_ramses_new_101's particle
    arrays are decoded on the device (ramses.read_parts) and never visit host
    memory.  Positions come out in [-0.5, 0.5) box units, as the reference's
    reader leaves them."""
    import torch
    t0 = time.perf_counter()
    r = ramses.read_parts(repository, version, family, scale_l, scale_t)
    torch.cuda.synchronize()
    times = {"read": (time.perf_counter() - t0) * 1e3}
    finder.configure(int(r["nselected"]), box=box, **(finder_params or {}))
    out = _run_device(r["pos"], r["vel"], r["mass"], box, hub, gravconst, epot, particle_views, times)
    out.update(ndm=r["ndm"], nstar=r["nstar"], nselected=r["nselected"])
    return out
