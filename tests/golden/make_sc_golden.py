"""Generate shrinking-sphere centre fixtures with the REFERENCE's own functions.

Runs det_mass_17, det_center_18 and refine_centers_1b with H.SC on
(CHP:1555-1596 -> det_halo_center_sphere_1b1, 1498-1541), then
compute_ang_mom_19, r_halos_1a and det_main_axis_1b2 about the refined centre,
on seeded synthetic halos; stores inputs and outputs in tests/golden/sc_case.npz.

Usage (where the reference is mounted): python tests/golden/make_sc_golden.py /path/to/reference
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

FIELDS = ["px", "py", "pz", "Lx", "Ly", "Lz", "r", "sha", "shb", "shc"]
DCELL_MIN = 2e-3
EPS_SC = 0.05


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
    H.SC = True
    H.dcell_min = np.float64(DCELL_MIN)
    H.eps_SC = np.float64(EPS_SC)
    H.cdm = False
    H.massp = 1.0
    sizes = [20, 80, 333, 1200, 5000, 700]
    rng = np.random.default_rng(71)
    off = [0]
    P, V, M, D = [], [], [], []
    for k, n in enumerate(sizes):
        o, p, v, m, d = synthetic.halo_catalogue(1, seed=500 + k, nmin=n, nmax=n + 1, box=box)
        if k == 5:  # across the periodic edge
            p = np.mod(p - p.mean(0) + np.array([-box / 2 + 0.01, box / 2 - 0.01, box / 2 - 0.01]) + box / 2,
                       box) - box / 2
        d = d * rng.uniform(0.9, 1.1, size=d.shape)  # densest member off the centre of mass
        m = m * rng.uniform(0.5, 1.5, size=m.shape)
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
        CHP.det_main_axis_1b2(rec, member=member)
        out[h] = [rec[f] for f in FIELDS]
    for name in list(H.mem.keys()):
        H.deallocate(name)
    np.savez_compressed(os.path.join(HERE, "sc_case.npz"), off=off, pos=pos, vel=vel, mass=mass, dens=dens,
                        out=out, fields=np.array(FIELDS), Lbox=box, Hub_pt=70.0, gravconst=430.1,
                        dcell_min=DCELL_MIN, eps_sc=EPS_SC)
    print("sc_case", nh, "halos", int(off[-1]), "members")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HALOMAKER_REF")
    if not root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> (or set HALOMAKER_REF)")
    main(root)
