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


_STAGE_BYTES = 256 << 20  # one pinned staging buffer of the upload


def upload(arrays, dev, stage_bytes: int = _STAGE_BYTES):
    """Copy host arrays (float64, any shape) to new device tensors through two
    pinned staging buffers: the host copy of one chunk into a staging buffer
    overlaps the upload of the previous chunk on a side stream, so the time is
    about the slower of the two copies instead of their sum (pinning a whole
    array first, then uploading it, pays both).  Returns the device tensors;
    the current stream waits for the uploads."""
    import torch
    side = torch.cuda.Stream(device=dev)
    per = max(1, stage_bytes // 8)
    stage = [torch.empty(per, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    done = [None, None]
    out = []
    k = 0
    for a in arrays:
        src = torch.from_numpy(np.ascontiguousarray(a, np.float64)).reshape(-1)
        dst = torch.empty(src.numel(), dtype=torch.float64, device=dev)
        for i in range(0, src.numel(), per):
            m = min(per, src.numel() - i)
            b = k & 1
            if done[b] is not None:
                done[b].synchronize()  # the upload that last read this buffer has finished
            stage[b][:m].copy_(src[i:i + m])
            with torch.cuda.stream(side):
                dst[i:i + m].copy_(stage[b][:m], non_blocking=True)
                done[b] = torch.cuda.Event()
                done[b].record(side)
            k += 1
        out.append(dst.reshape(a.shape))
    torch.cuda.current_stream(dev).wait_stream(side)
    for t in out:
        t.record_stream(side)
    return out


def run_snapshot(pos: np.ndarray, vel: np.ndarray, mass: np.ndarray, box: float = 1.0, hub: float = 70.0,
                 gravconst: float = 430.1, epot: int = 2, finder_params: dict | None = None,
                 particle_views: bool = False, ndm: int | None = None, cdm: bool = False, massp: float = 0.0,
                 virial: bool = True, vir_overdens: float = 178.0, rho_mean: float | None = None) -> dict:
    """Host arrays pos (N,3), vel (N,3), mass (N,) in box units ([-box/2, box/2)).

    Returns the structure selection (ids, tree arrays; the per-particle arrays
    whereIam_parts / pids_groupsorted only with particle_views), one property
    row per structure with members (halo_props.FIELDS, structure order =
    ascending id), with virial one row of the virial step per structure
    (halo_props.VIR_FIELDS), and per-stage times in ms (device stages by CUDA
    events, the rest by the host clock around synchronised steps).

    ndm: particles [0, ndm) are dark matter, the rest stars (det_mass_17's
    split; None: all dark matter); cdm: centre = member closest to the centre
    of mass; massp: dark-matter contamination threshold (H.massp);
    vir_overdens, rho_mean: H.vir_overdens and H.rho_mean of the virial step
    (CHP:1330-1331; rho_mean defaults to the total mass over box**3)."""
    import torch
    n = int(mass.shape[0])
    finder.configure(n, box=box, **(finder_params or {}))
    dev = torch.device("cuda")
    times = {}
    t0 = time.perf_counter()
    d_pos, d_vel, d_mass = upload((pos, vel, mass), dev)
    torch.cuda.synchronize()
    times["pin"] = 0.0  # staged: the host copies overlap the uploads
    times["h2d"] = (time.perf_counter() - t0) * 1e3
    opts = dict(ndm=ndm, cdm=cdm, massp=massp, virial=virial, vir_overdens=vir_overdens, rho_mean=rho_mean)
    return _run_device(d_pos, d_vel, d_mass, box, hub, gravconst, epot, particle_views, times, **opts)


def _run_device(d_pos, d_vel, d_mass, box, hub, gravconst, epot, particle_views, times, ndm=None, cdm=False,
                massp=0.0, virial=True, vir_overdens=178.0, rho_mean=None):
    """Finder, selection, member gather, properties and the virial step on
    device arrays."""
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
    gidx = msm.gather_index_device(gmass.shape[0], dev, stream=st) if ndm is not None else None
    torch.cuda.synchronize()
    times["gather"] = (time.perf_counter() - t0) * 1e3
    ns = int(ids.numel())
    out = torch.empty((max(ns, 1), halo_props.NF), dtype=torch.float64, device=dev)
    t0 = time.perf_counter()
    if ns:
        halo_props.compute_device(off, gpos, gvel, gmass, gdens, out, box, hub, gravconst, True, epot, stream=st,
                                  cdm=cdm, d_index=gidx, ndm=ndm, massp=massp)
    torch.cuda.synchronize()
    times["props"] = (time.perf_counter() - t0) * 1e3
    times["props_stages"] = halo_props.timings() if ns else {}
    vrows = None
    if virial and ns:
        # det_vir_1b on the same members (CHP:1241-1262), from the rows above
        t0 = time.perf_counter()
        rm = float(rho_mean) if rho_mean is not None else float(d_mass.sum().item()) / box ** 3
        vout = torch.empty((ns, halo_props.NV), dtype=torch.float64, device=dev)
        ep = "ep64" if epot & 1 else "ep32c"
        halo_props.virial_device(off, gpos, gvel, gmass, out, vout, box, hub, gravconst, vir_overdens, rm,
                                 ep=ep, stream=st)
        torch.cuda.synchronize()
        times["virial"] = (time.perf_counter() - t0) * 1e3
        vrows = vout.cpu().numpy()
    t0 = time.perf_counter()
    rows = out[:ns].cpu().numpy()
    ids_h = ids.cpu().numpy()
    off_h = off.cpu().numpy()
    times["d2h"] = (time.perf_counter() - t0) * 1e3
    return dict(sel, ids=ids_h, offsets=off_h, props=rows, virial=vrows, members=int(off_h[-1]) if ns else 0,
                timings=times)


def run_snapshot_files(repository, version: int = 3, family: str = "all", scale_l: float = 1.0,
                       scale_t: float = 1.0, box: float = 1.0, hub: float = 70.0, gravconst: float = 430.1,
                       epot: int = 2, finder_params: dict | None = None, particle_views: bool = False,
                       cdm: bool = False, massp: float = 0.0, virial: bool = True, vir_overdens: float = 178.0,
                       rho_mean: float | None = None) -> dict:
    """The same snapshot step starting from RAMSES part files (an
    output_NNNNN directory or the file paths): read_ramses_new_101's particle
    arrays are decoded on the device (ramses.read_parts) and never visit host
    memory.  Positions come out in [-0.5, 0.5) box units, as the reference's
    reader leaves them; dark-matter rows come first (family 'all'), so the
    reader's ndm splits dark matter from stars in the properties."""
    import torch
    t0 = time.perf_counter()
    r = ramses.read_parts(repository, version, family, scale_l, scale_t)
    torch.cuda.synchronize()
    times = {"read": (time.perf_counter() - t0) * 1e3}
    finder.configure(int(r["nselected"]), box=box, **(finder_params or {}))
    ndm = int(r["ndm"]) if family == "all" else (int(r["nselected"]) if family == "dm" else 0)
    out = _run_device(r["pos"], r["vel"], r["mass"], box, hub, gravconst, epot, particle_views, times, ndm=ndm,
                      cdm=cdm, massp=massp, virial=virial, vir_overdens=vir_overdens, rho_mean=rho_mean)
    out.update(ndm=r["ndm"], nstar=r["nstar"], nselected=r["nselected"])
    return out
