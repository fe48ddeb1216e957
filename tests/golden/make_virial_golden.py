"""Generate virial-property golden fixtures with the REFERENCE's own functions.

Runs the chain of _compute_halo_props (CHP:270-301) through det_vir_1b
(det_main_axis_1b2, det_halo_energies_1b3, det_vir_props_1b4 with
tab_props_inside_1b40 / potential_profile_1b40 under their default policies)
on seeded synthetic halos and stores inputs and outputs in
tests/golden/virial_case.npz.

Half of the halos get velocities scaled so that 2K is close to |W| (the
virial-theorem branch of det_vir_props_1b4), the others are left hot (the
overdensity fallback).  Sizes straddle the 1000-member limit of the direct
potential, so both normalisations of the potential profile are exercised.

Usage (where the reference is mounted): python tests/golden/make_virial_golden.py /path/to/reference
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

FIELDS = ["m", "px", "py", "pz", "vx", "vy", "vz", "r", "sha", "shb", "shc", "ek", "ep", "et", "rvir", "mvir",
          "cvel", "tvir", "rho_0", "r_c", "amax", "bmax", "cmax"]
VIR_OVERDENS = 178.0
RHO_MEAN = 2.0e-3


def main(refroot):
    sys.path.insert(0, os.path.join(refroot, "src"))
    sys.path.insert(0, os.path.join(REPO, "halomaker-python_b200"))
    import halo_defs as H
    H.FORTRAN = False
    import compute_halo_props as CHP
    from ahop_b200 import synthetic

    box = 100.0
    H.Lbox_pt = box
    H.Lbox_pt2 = box / 2
    H.FlagPeriod = 1
    H.Hub_pt = 70.0
    H.gravconst = np.float64(430.1)
    H.mode = "full"
    H.stellar_payload = False
    H.method = "MSM"
    H.DPMMC = False
    H.SC = False
    H.cdm = False
    H.massp = 1.0
    H.ANG_MOM_OF_R = False
    H.vir_overdens = np.float64(VIR_OVERDENS)
    H.rho_mean = np.float64(RHO_MEAN)
    sizes = [20, 64, 200, 500, 999, 1000, 1800, 4000, 300, 2500]
    rng = np.random.default_rng(57)
    off = [0]
    P, V, M, D = [], [], [], []
    G = 430.1
    for k, n in enumerate(sizes):
        o, p, v, m, d = synthetic.halo_catalogue(1, seed=300 + k, nmin=n, nmax=n + 1, box=box)
        if k == 8:  # across the periodic edge
            p = np.mod(p - p.mean(0) + np.array([box / 2 - 0.02, -box / 2 + 0.02, 0.0]) + box / 2, box) - box / 2
        m = m * rng.uniform(0.5, 1.5, size=m.shape)
        # velocity scale: close to virial for even k, hot for odd k
        c = p.mean(0)
        dr = p - c
        i, j = np.triu_indices(len(m), 1)
        W = -G * np.sum(m[i] * m[j] / np.sqrt(np.sum((dr[i] - dr[j]) ** 2, 1)))
        u = v - np.sum(m[:, None] * v, 0) / m.sum()
        K = 0.5 * np.sum(m * np.sum(u * u, 1))
        s = np.sqrt(-W / (2 * K)) * (rng.uniform(0.85, 1.1) if k % 2 == 0 else 3.0)
        v = u * s + rng.normal(size=3)
        P.append(p); V.append(v); M.append(m); D.append(d)
        off.append(off[-1] + len(m))
    pos = np.concatenate(P); vel = np.concatenate(V); mass = np.concatenate(M); dens = np.concatenate(D)
    off = np.array(off, np.int64)
    nh = len(sizes)
    H.ndm = len(mass)
    H.allocate("pos_10", (1, 3), np.float64)
    out = np.zeros((nh, len(FIELDS)))
    for h in range(nh):
        a, b = off[h], off[h + 1]
        member = (np.int32(b - a), np.arange(a, b), pos[a:b].copy(), vel[a:b].copy(), mass[a:b].copy(),
                  dens[a:b].copy())
        rec = np.zeros(1, dtype=H.halo_dtype)[0]
        rec["nmem"] = b - a
        CHP.det_mass_17(rec, member=member)
        CHP.det_center_18(rec, member=member)
        CHP.refine_centers_1b(rec, member=member)
        CHP.compute_ang_mom_19(rec, member=member)
        CHP.r_halos_1a(rec, member=member)
        d, v = CHP.det_main_axis_1b2(rec, member=member)
        CHP.det_halo_energies_1b3(rec, member=member)
        amax, bmax, cmax = CHP.det_vir_props_1b4(rec, v, member=member)
        vals = {f: rec[f] for f in FIELDS if f not in ("amax", "bmax", "cmax")}
        vals.update(amax=amax, bmax=bmax, cmax=cmax)
        out[h] = [vals[f] for f in FIELDS]
    for name in list(H.mem.keys()):
        H.deallocate(name)
    np.savez_compressed(os.path.join(HERE, "virial_case.npz"), off=off, pos=pos, vel=vel, mass=mass, dens=dens,
                        out=out, fields=np.array(FIELDS), Lbox=box, Hub_pt=70.0, gravconst=430.1,
                        vir_overdens=VIR_OVERDENS, rho_mean=RHO_MEAN, nshell=1000)
    print("virial_case", nh, "halos", int(off[-1]), "members")
    for h in range(nh):
        print(sizes[h], dict(zip(["rvir", "mvir", "ep", "et"], out[h, [14, 15, 12, 13]])))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HALOMAKER_REF")
    if not root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> (or set HALOMAKER_REF)")
    main(root)
