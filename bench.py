"""Benchmark: AdaptaHOP end to end on one B200 per rank (replicas), JSON line out.

Workload (N=1): the 256^3 box -- 16,777,216 float64 DM particles from the
seeded clustered generator (19,200 NFW halos with subhalos, counts 20..2e6,
plus 40 % uniform background), nvoisins=32, nhop=16, rhot=80, fudge=4,
fudgepsilon=1e-5, alphap=1, nmembthresh=20.

  value  -- Mparticles/s of the full pipeline with pos/mass already in HBM
            (ahop_compute_adaptahop_device), CUDA events on the compute stream;
  e2e    -- the same metric through the public drop-in call
            compute_adaptahop.neikdtree.compute_adaptahop(pos, mass) on host
            buffers: host->device copies, all stages and the copy-back of the
            module outputs inside the timed region;
  roofline -- the fused kNN + density kernel (the dominant kernel) against the
            measured HBM copy bandwidth;
  cpu_baseline -- the CPU restatement of the reference finder (OpenMP, all host
            cores): one full pass over the same 256^3 box.

--impl reference times that CPU restatement (the reference's own Fortran
cannot be built: no Fortran compiler in the image) on the same 256^3 box, one
full finder pass per timed step; its warm-up steps run the 64^3 box of the same
generator (the CPU path has no caches or compiled code to warm beyond its
thread pool, and a full pass takes tens of seconds).
Multi-GPU: the finder does not shard (its structure tree needs a global
merge), so --gpus N runs N independent replicas (weak scaling).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "halomaker-python_b200"))

METRIC = "Mpart/s end-to-end vs host CPU; halo Epot pairs/s FP32-comp vs FP64 at 1e-6"
PARAMS = dict(nvoisins=32, nhop=16, rho_threshold=80.0, fudge=4.0, fudgepsilon=1e-5, alphap=1.0, nmembthresh=20)
WORKLOAD = dict(name="c2_256cubed", npart=16_777_216, nhalo=19_200, seed=2, nmin=20, nmax=2_000_000)
WARM_SAMPLE = dict(name="64cubed_same_generator", npart=262_144, nhalo=300, seed=2, nmax=31_250)

# ncu counters of knn_leaf_kernel (DRAM read + write bytes and warp
# instructions, per particle) from the capture summarised in
# profiles/knn_leaf_kernel_8m.md; the bench line scales them to the workload.
# They are re-measured whenever the kernel changes.
NCU_KNN = dict(profiled="knn_leaf_kernel, 8,000,000-particle clustered box, one launch",
               dram_bytes_per_particle=225.694848, warp_instructions_per_particle=3750.793200)


def _gen(spec):
    from ahop_b200 import synthetic
    return synthetic.clustered_box(spec["npart"], spec["nhalo"], seed=spec["seed"], nmax=spec["nmax"])


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload_config(spec, world):
    """The bench line's config; both arms print the same one."""
    # change_pos_1310: epsilon = fudgepsilon * xlong / npart**(1/3)
    eps = PARAMS["fudgepsilon"] * 1.0 / spec["npart"] ** (1.0 / 3.0)
    return {"workload": spec["name"], "npart": spec["npart"], "nhalo": spec["nhalo"], "seed": spec["seed"],
            "epsilon": eps, **PARAMS, "l2": f"inputs ({spec['npart'] * 32 / 1e6:.0f} MB) larger than L2",
            "parallelism": f"replicas{world}"}


def cpu_rate(ps, nthreads=None):
    """Oracle (CPU restatement, OpenMP) Mparticles/s of one full finder pass."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    prm = oracle.default_params(ps.n, nthreads=nthreads or os.cpu_count(),
                                **{k: PARAMS[k] for k in ("nvoisins", "nhop", "rho_threshold", "fudge", "alphap",
                                                          "nmembthresh")})
    t = time.perf_counter()
    r = oracle.run(ps.pos, ps.mass, prm)
    dt = time.perf_counter() - t
    return ps.n / dt / 1e6, dt, prm["nthreads"], r


def run_reference(args, rank, world):
    """The CPU path on the bench workload: K full passes over the 256^3 box,
    after W warm-up passes over the 64^3 box of the same generator."""
    if rank != 0:
        return
    warm = _gen(WARM_SAMPLE)
    for _ in range(args.warmup):
        cpu_rate(warm)
    del warm
    spec = dict(WORKLOAD)
    if args.npart:
        spec = _scaled(spec, args.npart)
    ps = _gen(spec)
    secs = []
    nth = os.cpu_count()
    for _ in range(args.steps):
        _, dt, nth, _ = cpu_rate(ps)
        secs.append(dt)
    tot = sum(secs)
    v = ps.n * len(secs) / tot / 1e6
    sample = (f"{ps.n} particles ({spec['name']}, {spec['nhalo']} halos, seed {spec['seed']}): the full bench box, "
              f"one full finder pass per timed step ({min(secs):.1f}-{max(secs):.1f} s); warm-up passes on "
              f"{WARM_SAMPLE['npart']} particles ({WARM_SAMPLE['name']})")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "Mpart/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / len(secs) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(spec, world),
            "cpu_baseline": {"value": v, "unit": "Mpart/s", "cores": nth, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "Mpart/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _scaled(spec, npart):
    return dict(spec, npart=npart, nhalo=max(10, int(spec["nhalo"] * npart / spec["npart"])),
                name=f"scaled_{npart}")


def halo_section(args, torch, dist=None):
    """Batched direct-sum potential: FP32-compensated vs FP64 forms on the GPU.

    Workload: 20,000 halos with member counts from dN/dn ~ n^-1.9 on
    [20, 2e6] (seed 3), NFW positions (c=10) and Gaussian velocities in a
    100-unit periodic box; pairs = sum n(n-1)/2.  Each form is timed alone
    (CUDA events around its persistent pair kernel) over the same work list.
    With several ranks the halos are split into contiguous runs of equal cost,
    each rank times its own run and the slowest rank's time counts (the
    catalogue is fixed: strong scaling); rank 0 gathers the E_pot rows.
    """
    import numpy as np
    from ahop_b200 import halo_props, replicas, synthetic
    off, pos, vel, mass, dens = synthetic.halo_catalogue(args.nhalo, seed=args.halo_seed, nmin=20,
                                                         nmax=args.halo_nmax, box=100.0)
    if args.tiles:
        halo_props.set_tiles([args.tiles] * halo_props.BUCKETS)
    world = dist.get_world_size() if dist is not None and dist.is_initialized() else 1
    nh_all = len(off) - 1
    if world > 1:
        b = replicas.partition_halos(off, world)
        off, m0, m1 = replicas.local_members(off, b, dist.get_rank())
        pos, vel, mass, dens = pos[m0:m1], vel[m0:m1], mass[m0:m1], dens[m0:m1]
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    d_off, d_pos, d_vel, d_mass, d_dens = t(off), t(pos), t(vel), t(mass), t(dens)
    nh = len(off) - 1
    out = torch.zeros((nh, halo_props.NF), dtype=torch.float64, device=dev)
    st = torch.cuda.current_stream()
    # the first call also runs the tile autotuner (per halo-size bucket)
    halo_props.compute_device(d_off, d_pos, d_vel, d_mass, d_dens, out, 100.0, 70.0, epot=3, stream=st)
    tune_ms = halo_props.timings()["tune_ms"]
    o = out.cpu().numpy()
    ep64, ep32 = o[:, halo_props.FIELDS.index("ep64")], o[:, halo_props.FIELDS.index("ep32c")]
    ok = ep64 != 0
    rel = float(np.max(np.abs(ep32[ok] - ep64[ok]) / np.abs(ep64[ok])))
    t64, t32 = [], []
    for _ in range(max(1, args.steps)):
        # one call runs both forms back to back in its captured graph; CUDA
        # events bracket each persistent pair kernel
        halo_props.compute_device(d_off, d_pos, d_vel, d_mass, d_dens, out, 100.0, 70.0, epot=3, stream=st)
        tm = halo_props.timings()
        t64.append(tm["epot64"])
        t32.append(tm["epot32c"])
    if world > 1:
        rows = np.stack([ep64, ep32], 1)
        full = replicas.gather_rows(rows, b, dist)
        if full is not None:
            ok = full[:, 0] != 0
            rel = float(np.max(np.abs(full[ok, 1] - full[ok, 0]) / np.abs(full[ok, 0])))
        t64 = [replicas.max_over_ranks(x, dist) for x in t64]
        t32 = [replicas.max_over_ranks(x, dist) for x in t32]
    # virial step (det_vir_1b: 1000 ellipsoidal shells per halo) on the FP64 rows
    halo_props.compute_device(d_off, d_pos, d_vel, d_mass, d_dens, out, 100.0, 70.0, epot=1, stream=st)
    vout = torch.zeros((nh, halo_props.NV), dtype=torch.float64, device=dev)
    tv = []
    for _ in range(max(1, args.steps)):
        halo_props.virial_device(d_off, d_pos, d_vel, d_mass, out, vout, 100.0, 70.0, 430.1, 178.0, 2e-3,
                                 stream=st)
        tv.append(halo_props.virial_last_ms())
    pairs = float(tm["pairs"])
    if world > 1:
        tv = [replicas.max_over_ranks(x, dist) for x in tv]
        import torch as _t
        pt = _t.tensor([pairs], dtype=_t.float64, device=dev)
        dist.all_reduce(pt)
        pairs = float(pt.item())
    m64, m32 = statistics.mean(t64), statistics.mean(t32)
    nominal_fp32 = 148 * 128 * 2 * 1.965e9 / 1e12  # TFLOP/s, non-tensor FP32 at max clock
    mufu_peak = 148 * 16 * 1.965e9 / 1e12           # T reciprocal square roots/s
    rate32 = pairs / (m32 / 1e3)
    return {"workload": f"{nh_all} halos, counts n^-1.9 on [20, {args.halo_nmax:g}], seed {args.halo_seed}"
                        + (f", split over {world} ranks by cost" if world > 1 else ""),
            "pairs": pairs, "fp64_ms": m64, "fp32c_ms": m32,
            "fp64_pairs_per_s": pairs / (m64 / 1e3), "fp32c_pairs_per_s": rate32,
            "fp32c_over_fp64": m64 / m32, "max_rel_err_fp32c_vs_fp64": rel, "tolerance": 1e-6,
            # the compensated form takes one approximate reciprocal square root
            # per pair on the MUFU pipe (16 results per SM per cycle) and, per
            # pair, 7 FP32 lane operations for far pairs (3 separation, 3 r^2,
            # 1 mass-weighted accumulation) or 13 for near ones (hi/lo
            # separation), packed two per f32x2 instruction on 128 FP32 lanes
            # per SM per cycle; far pairs are therefore MUFU-bound.  The fp32c
            # time includes the Morton sort of the members.  The 20 flop/pair
            # convention is kept beside it.
            "roofline": {"bound": "MUFU pipe (rsqrt)", "rsqrt_per_pair": 1, "achieved": rate32 / 1e12,
                         "peak": mufu_peak, "unit": "T rsqrt/s", "frac": rate32 / 1e12 / mufu_peak,
                         "peak_source": "nominal (148 SMs x 16 MUFU results/clk x 1.965 GHz)",
                         "fp32_lane_ops_per_pair": "7 far, 13 near",
                         "tflops_at_20_flop_per_pair": 20 * rate32 / 1e12,
                         "tflops_peak_nominal": nominal_fp32},
            "moments_ms": tm["moments"], "items": int(tm["items"]), "tile_rows_per_bucket": halo_props.tiles()["rows"],
            "autotune_ms": tune_ms, "graph_replays": int(tm["graph_replays"]), "virial_ms": statistics.mean(tv),
            "virial_members_per_s": float(off[-1]) * world / (statistics.mean(tv) / 1e3)}


def reader_section(args):
    """RAMSES part files -> device arrays: the device reader (record walk,
    one read per file into pinned memory, payload copies, family count and
    scatter kernels) against the CPU restatement of the reference's reader
    (NumPy, one thread).  The files were just written, so they are read from
    the page cache: this times decoding, not the disk."""
    import tempfile
    import numpy as np
    import torch
    from ahop_b200 import build, ramses, synthetic
    sys.path.insert(0, os.path.join(REPO, "tests", "golden"))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ramses_files
    import ramses_oracle
    build.build()
    ps = synthetic.workload(args.reader)
    n = ps.n
    star = ps.mass < 0.5 * ps.mass.max()
    ids = np.empty(n, np.int32)
    ids[~star] = np.arange(1, int((~star).sum()) + 1)
    ids[star] = np.arange(1, int(star.sum()) + 1)
    kind = np.where(star, 2, 1).astype(np.int8)
    P = dict(pos=ps.pos + 0.5, vel=ps.vel, mass=ps.mass, id=ids, fam=kind, kind=kind,
             tbirth=np.zeros(n), level=np.zeros(n, np.int32), metal=np.zeros(n))
    ncpu = 64
    bounds = np.linspace(0, n, ncpu + 1).astype(np.int64)
    res = {"mode": "reader", "workload": args.reader, "npart": n, "stars": int(star.sum()), "files": ncpu,
           "format": "Ra4"}
    with tempfile.TemporaryDirectory() as tmp:
        paths = ramses_files.write_arrays(tmp, P, 4, bounds)
        res["bytes"] = int(sum(os.path.getsize(p) for p in paths))
        walls = []
        for i in range(args.warmup + max(1, args.steps)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            r = ramses.read_parts(paths, 4, "all", 1.0, 1.0)
            torch.cuda.synchronize()
            if i >= args.warmup:
                walls.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        o = ramses_oracle.read_parts(paths, 4, "all", 1.0, 1.0)
        cpu_s = time.perf_counter() - t0
        same = all(np.array_equal(r[k].cpu().numpy(), o[k]) for k in ("pos", "vel", "mass"))
    res.update(device_s=walls, device_Mpart_per_s=n / min(walls) / 1e6, device_GB_per_s=res["bytes"] / min(walls) / 1e9,
               cpu_s=cpu_s, cpu_Mpart_per_s=n / cpu_s / 1e6, cpu_cores=1, cpu_kind="port (NumPy)",
               identical_to_cpu=bool(same))
    return res


def pipeline_section(args):
    """Whole snapshots on one GPU: W untimed + K timed runs of
    pipeline.run_snapshot (finder, MSM selection, member gather, properties,
    virial step); per-stage times of the last run and the mean particles/s
    over the timed runs (host clock around the synchronised call, pinned host
    arrays in, property rows out).  With --check, the finder's outputs are
    compared with the CPU restatement of the reference on the same particles,
    which is timed beside."""
    import numpy as np
    from ahop_b200 import build, halo_props, pipeline, synthetic
    build.build()
    t0 = time.perf_counter()
    ps = synthetic.workload(args.pipeline)
    gen_s = time.perf_counter() - t0
    kw = dict(box=ps.box, epot=2, ndm=ps.ndm)
    for _ in range(args.warmup):
        pipeline.run_snapshot(ps.pos, ps.vel, ps.mass, **kw)
    walls = []
    res = None
    for _ in range(max(1, args.steps)):
        t0 = time.perf_counter()
        res = pipeline.run_snapshot(ps.pos, ps.vel, ps.mass, **kw)
        walls.append(time.perf_counter() - t0)
    t = res["timings"]
    stars = int(np.count_nonzero(ps.mass < ps.mass.max() * 0.5)) if ps.n else 0
    check = None
    if args.check:
        # the finder's outputs through the drop-in on the same particles
        # against the CPU restatement of the reference (OpenMP, all host cores)
        from ahop_b200 import finder
        finder.configure(ps.n)
        t0 = time.perf_counter()
        out = finder.run(ps.pos, ps.mass)
        gpu_s = time.perf_counter() - t0
        rate, cpu_s, nth, ref = cpu_rate(ps)
        check = {"density_equal": bool(np.array_equal(out["density"], ref["density"])),
                 "liste_parts_equal": bool(np.array_equal(out["liste_parts"], ref["liste_parts"])),
                 "integer_table_equal": bool(np.array_equal(out["integer_table"], ref["integer_table"])),
                 "real_table_equal": bool(np.array_equal(out["real_table"], ref["real_table"])),
                 "nnodes": int(out["nnodes"]), "oracle_nnodes": int(ref["nnodes"]),
                 "gpu_finder_e2e_s": gpu_s, "cpu_finder_s": cpu_s, "cpu_Mpart_per_s": rate, "cpu_cores": nth,
                 "cpu_kind": "port (C++/OpenMP restatement of the reference finder)"}
    return {"mode": "pipeline", "workload": args.pipeline, "npart": ps.n, "stars": stars, "generate_s": gen_s,
            "check": check,
            "steps": len(walls), "warmup": args.warmup, "wall_s": walls, "Mpart_per_s": ps.n / min(walls) / 1e6,
            "nstruct": int(res["nstruct"]), "nb_of_halos": int(res["nb_of_halos"]),
            "structures_with_members": int(len(res["ids"])), "members": int(res["members"]),
            "stage_ms": {k: v for k, v in t.items() if not isinstance(v, dict)},
            "finder_stages_ms": {k: v for k, v in t["finder_stages"].items()},
            "props_stages": t["props_stages"], "tile_rows_per_bucket": halo_props.tiles()["rows"]}


def adjoint_section(args):
    """Differentiation on the 2,097,152-particle box (2,000 NFW halos of up
    to ~74,000 members, seed 4): forward and backward of the SPH density with
    the finder's 32-neighbour lists held fixed, and of the per-halo
    direct-sum potential over the generator's halos (members grouped by
    halo); CUDA events around each call, W untimed + K timed repeats."""
    import numpy as np
    import torch
    from ahop_b200 import autograd, build, finder, synthetic
    build.build()
    ps = synthetic.workload("c4_2m")
    finder.configure(ps.n)
    st = finder.run_stages(ps.pos, ps.mass, last_stage=2, store_neighbours=32)
    dev = torch.device("cuda")
    pos = torch.from_numpy(ps.pos).to(dev)
    mass = torch.from_numpy(ps.mass).to(dev)
    nei = torch.from_numpy(np.ascontiguousarray(st["neighbours"] - 1, np.int32)).to(dev)
    order = np.argsort(ps.halo_id, kind="stable")
    order = order[ps.halo_id[order] >= 0]
    counts = np.bincount(ps.halo_id[order])
    off = torch.from_numpy(np.concatenate([[0], np.cumsum(counts)]).astype(np.int64))
    hpos = torch.from_numpy(np.ascontiguousarray(ps.pos[order])).to(dev)
    hmass = torch.from_numpy(np.ascontiguousarray(ps.mass[order])).to(dev)
    g = torch.randn(ps.n, dtype=torch.float64, device=dev)

    def timed(fn):
        for _ in range(args.warmup):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ms = []
        for _ in range(max(1, args.steps)):
            torch.cuda.synchronize()
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        return statistics.mean(ms)

    def dens_fwd():
        autograd.density_fixed(pos, mass, nei, 1.0)

    def dens_bwd():
        p = pos.clone().requires_grad_(True)
        (autograd.SPHDensity.apply(p, mass, nei, 1.0) * g).sum().backward()

    def pot_fwd():
        autograd.HaloPotential.apply(hpos, hmass, off, 1.0, 430.1)

    def pot_bwd():
        p = hpos.clone().requires_grad_(True)
        autograd.HaloPotential.apply(p, hmass, off, 1.0, 430.1).sum().backward()

    f_d, b_d, f_p, b_p = timed(dens_fwd), timed(dens_bwd), timed(pot_fwd), timed(pot_bwd)
    pairs = float((counts.astype(np.float64) * (counts - 1) / 2).sum())
    return {"mode": "adjoint", "workload": "c4_2m", "npart": ps.n, "nhalo": len(counts),
            "halo_members": int(counts.sum()), "pairs": pairs, "density_forward_ms": f_d,
            "density_forward_and_backward_ms": b_d, "potential_forward_ms": f_p,
            "potential_forward_and_backward_ms": b_p,
            "density_backward_Mpart_per_s": ps.n / ((b_d - f_d) / 1e3) / 1e6,
            "potential_backward_pairs_per_s": pairs / ((b_p - f_p) / 1e3)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--npart", type=int, default=0, help="override the workload size (testing)")
    ap.add_argument("--no-halo", action="store_true", help="skip the batched halo E_pot section")
    ap.add_argument("--nhalo", type=int, default=20000, help="halos in the E_pot section")
    ap.add_argument("--halo-nmax", type=int, default=2_000_000, help="largest halo count of the E_pot catalogue")
    ap.add_argument("--halo-seed", type=int, default=3, help="seed of the E_pot catalogue")
    ap.add_argument("--tiles", type=int, default=0, choices=[0, 128, 256, 512],
                    help="pin the FP32 pair kernel's rows per item in every bucket (0: autotune)")
    ap.add_argument("--halo-only", action="store_true",
                    help="run only the batched halo section and print its JSON (profiling; not the bench line)")
    ap.add_argument("--reader", default="", metavar="WORKLOAD",
                    help="write a named synthetic workload as RAMSES Ra4 part files (64 files, in a temporary "
                         "directory) and time the device reader against the CPU restatement (not the bench line)")
    ap.add_argument("--check", action="store_true",
                    help="with --pipeline: compare the finder's outputs with the CPU restatement of the reference "
                         "on the same particles and time it beside")
    ap.add_argument("--adjoint", action="store_true",
                    help="time the density and potential adjoints on the 2,097,152-particle box (not the bench line)")
    ap.add_argument("--pipeline", default="", metavar="WORKLOAD",
                    help="run whole snapshots (finder, MSM, member gather, FP32-compensated properties) on a named "
                         "synthetic workload (e.g. c5_512cubed) and print per-stage times (not the bench line)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.pipeline:
        print(json.dumps(pipeline_section(args)))
        return
    if args.adjoint:
        print(json.dumps(adjoint_section(args)))
        return
    if args.reader:
        print(json.dumps(reader_section(args)))
        return
    if args.halo_only:
        from ahop_b200 import build
        build.build()
        res = halo_section(args, torch, dist if world > 1 else None)
        if rank == 0:
            print(json.dumps(res))
        if world > 1:
            dist.destroy_process_group()
        return

    from ahop_b200 import _lib as L, finder, build
    from compute_adaptahop import neikdtree
    build.build()
    spec = dict(WORKLOAD)
    if args.npart:
        spec = _scaled(spec, args.npart)
    ps = _gen(spec)
    n = ps.n
    eps = finder.configure(n, **PARAMS)
    lib = L.lib()
    # device-resident inputs (Fortran pos(3,n) layout == (n,3) row-major)
    d_pos = torch.from_numpy(ps.pos).cuda()
    d_mass = torch.from_numpy(ps.mass).cuda()
    stream = torch.cuda.current_stream()

    def dev_step():
        L.check(lib.ahop_compute_adaptahop_device(d_pos.data_ptr(), d_mass.data_ptr(), n, C.c_void_p(stream.cuda_stream)),
                "compute_device")

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(args.warmup):
        dev_step()
    torch.cuda.synchronize()
    knn_ms, stage = [], []
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            dev_step()
            t = L.timings()
            knn_ms.append(t["knn_kernel"])
            stage.append(t)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
    dev_ms = e0.elapsed_time(e1)
    if world > 1:
        tt = torch.tensor([dev_ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dev_ms = float(tt.item())
    value = world * n * args.steps / (dev_ms / 1e3) / 1e6

    # end to end through the public drop-in call on pinned host buffers
    pos_h = torch.from_numpy(ps.pos).pin_memory().numpy()
    mass_h = torch.from_numpy(ps.mass).pin_memory().numpy()
    neikdtree.compute_adaptahop(pos_h.T, mass_h)  # warm
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        neikdtree.compute_adaptahop(pos_h.T, mass_h)
        _ = int(neikdtree.nnodes)
    e2e_s = time.perf_counter() - t0
    if world > 1:
        tt = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e = world * n * args.steps / e2e_s / 1e6
    nnodes = int(neikdtree.nnodes)
    d2h = n * 8 + neikdtree.liste_parts.nbytes + nnodes * (64 + 24)
    h2d = n * 32

    # roofline of the fused kNN + density kernel: 168 algorithmic bytes per particle
    knn_avg = statistics.mean(knn_ms)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(REPO, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    alg = 168.0 * n
    achieved = alg / (knn_avg / 1e3) / 1e9
    traffic = NCU_KNN["dram_bytes_per_particle"] * n
    inst = NCU_KNN["warp_instructions_per_particle"]
    roof = {"kernel": "knn_leaf_kernel", "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "alg_bytes_per_launch": alg,
            "launch_ms": knn_avg, "peak_source": "measured" if peaks else "fallback",
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per particle x n (" +
                              NCU_KNN["profiled"] + ")"}
    if inst:
        # the kernel is bound by instruction issue, not HBM: the warp instructions
        # ncu counted per query (profiles/) over this launch's time, against the
        # issue peak of 4 warp schedulers per SM at the SM clock seen
        props = torch.cuda.get_device_properties(local)
        mhz = clk.summary().get("sm_mhz") or 1965.0
        issue_peak = props.multi_processor_count * 4 * mhz * 1e6
        ach = inst * n / (knn_avg / 1e3)
        roof["issue"] = {"achieved_warp_inst_per_s": ach, "peak_warp_inst_per_s": issue_peak,
                         "frac": ach / issue_peak, "warp_inst_per_query": inst}
    # kNN and structure-tree counters come from one more call, after the timed
    # region, with the profiling instances of the kernels (the timed calls run
    # the production instances, which count nothing)
    lib.ahop_debug_set_task_profile.argtypes = [C.c_int32]
    L.check(lib.ahop_debug_set_task_profile(1), "set_task_profile")
    dev_step()
    torch.cuda.synchronize()
    L.check(lib.ahop_debug_set_task_profile(0), "set_task_profile")
    ts = (C.c_int64 * 30)()
    lib.ahop_debug_tree_stats(ts, 30)
    tree_stats = {"structural_Mcycles": ts[0] / 1e6, "level_stats_Mcycles": ts[1] / 1e6,
                  "exact_Mcycles": ts[2] / 1e6, "levels": ts[3], "undecided_exact_passes": ts[4],
                  "max_levels_one_task": ts[5], "max_Mcycles_one_task": ts[6] / 1e6,
                  "structural_passes": ts[7]}
    nql = max(1, ts[8])
    knn_stats = {"query_leaves": ts[8], "cand_leaves_per_query_leaf": ts[9] / nql,
                 "leaf_visits_per_query": ts[10] / n, "insertions_per_query": ts[11] / n, "overflow_leaves": ts[12],
                 "ideal_visits_per_query": ts[18] / n, "chunks_per_query": ts[26] / n,
                 "ballot_hits_per_query": ts[27] / n,
                 "union_visits_per_query_leaf": ts[28] / max(1, ts[29]),
                 "overflow_cycle_share": ts[19] / max(1, ts[19] + ts[20])}
    ph = [float(ts[21 + k]) for k in range(5)]
    if sum(ph) > 0:
        knn_stats["cycle_share"] = {k: v / sum(ph) for k, v in zip(
            ("bound_and_seed_sort", "candidates_and_sort", "seed_lists", "scan", "density"), ph)}
    mean_stage = {k: statistics.mean(s[k] for s in stage) for k in
                  ("tree", "knn_density", "hop_groups", "saddles", "nodes", "membership", "total")}
    line = {"metric": METRIC, "value": value, "unit": "Mpart/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(spec, world),
            "e2e": {"value": e2e, "unit": "Mpart/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": roof, "stages_ms": mean_stage,
            "stages_mpart_per_s": {k: (n / (v / 1e3) / 1e6 if v > 0 else None) for k, v in mean_stage.items()},
            "gpu_launches": int(stage[-1]["kernel_launches"]) * args.steps,
            "cub_calls_per_step": int(stage[-1]["cub_calls"]), "tree_waves": int(stage[-1]["tree_waves"]),
            "nnodes": nnodes, "tree_stats": tree_stats, "knn_stats": knn_stats, "clocks": clk.summary()}
    if not args.no_halo:
        line["halo_epot"] = halo_section(args, torch, dist if world > 1 else None)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, dt, nth, _ = cpu_rate(ps)
        line["cpu_baseline"] = {"value": rate, "unit": "Mpart/s", "cores": nth, "kind": "port",
                                "sample": f"{n} particles ({spec['name']}, the bench box): one full finder pass, "
                                          f"{dt:.1f} s"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    neikdtree.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
