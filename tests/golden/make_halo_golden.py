"""Generate per-halo property golden fixtures with the REFERENCE's own functions.

Runs src/compute_halo_props.py's per-halo reductions -- det_mass_17,
det_center_18, refine_centers_1b, compute_ang_mom_19, r_halos_1a,
det_main_axis_1b2, det_halo_energies_1b3 and compute_spin_parameter_1c, the
chain of _compute_halo_props (CHP:270-301) up to the virial step -- on seeded
synthetic halos and stores inputs and outputs in tests/golden/halo_case.npz.

Halos with fewer than 1000 members get the reference's direct pair-sum
potential (CHP:1413-1427); larger ones get its ellipsoid formula
(CHP:1405-1412), which the batched kernel does not compute (it sums pairs for
every size), so for those only the O(n) fields are compared.

A second case (halo_case_stars.npz) runs the same chain in mode 'full' with
H.cdm = True on halos that hold stars (particle indices at or above H.ndm) and
contaminating heavy dark-matter members: det_mass_17's ndm, nstar, mdm, m*,
mcontam (CHP:766-780), det_center_18's centre of mass and closest member
(CHP:917-934) and its sigma_dm / sigma* (CHP:962-966).

Usage (where the reference is mounted): python tests/golden/make_halo_golden.py /path/to/reference
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

FIELDS = ["m", "px", "py", "pz", "vx", "vy", "vz", "Lx", "Ly", "Lz", "r", "sha", "shb", "shc", "ek", "ep",
          "et", "spin", "sigma"]
STAR_FIELDS = FIELDS + ["ndm", "nstar", "mdm", "m*", "mcontam", "sigma_dm", "sigma*"]


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
    sizes = [20, 57, 150, 420, 999, 1500, 3000]
    rng = np.random.default_rng(31)
    off = [0]
    P, V, M, D = [], [], [], []
    for k, n in enumerate(sizes):
        o, p, v, m, d = synthetic.halo_catalogue(1, seed=100 + k, nmin=n, nmax=n + 1, box=box)
        # one halo straddles the periodic boundary
        if k == 2:
            p = np.mod(p - p.mean(0) + np.array([box / 2 - 0.05, 0.0, -box / 2 + 0.05]) + box / 2, box) - box / 2
        m = m * rng.uniform(0.5, 1.5, size=m.shape)
        P.append(p); V.append(v); M.append(m); D.append(d)
        off.append(off[-1] + len(m))
    pos = np.concatenate(P); vel = np.concatenate(V); mass = np.concatenate(M); dens = np.concatenate(D)
    off = np.array(off, np.int64)
    nh = len(sizes)
    H.ndm = len(mass)  # all members are dark matter
    H.allocate("pos_10", (1, 3), np.float64)  # referenced by det_center_18
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
        CHP.det_halo_energies_1b3(rec, member=member)
        CHP.compute_spin_parameter_1c(rec)
        out[h] = [rec[f] for f in FIELDS]
    np.savez_compressed(os.path.join(HERE, "halo_case.npz"), off=off, pos=pos, vel=vel, mass=mass, dens=dens,
                        out=out, fields=np.array(FIELDS), Lbox=box, Hub_pt=70.0, gravconst=430.1)
    print("halo_case", nh, "halos", int(off[-1]), "members")

    # stars and contamination, centre of mass (cdm)
    H.cdm = True
    H.massp = 0.8
    ndm = 1_000_000
    index = np.empty(len(mass), np.int64)
    mass2 = mass.copy()
    for h in range(nh):
        a, b = off[h], off[h + 1]
        k = b - a
        star = rng.random(k) < 0.3
        # particle ids: dark matter below ndm, stars at or above it (indexps < H.ndm is the mask)
        index[a:b] = np.where(star, ndm + rng.integers(0, 10**6, k), rng.integers(0, ndm, k))
        mass2[a:b] = np.where(star, 0.1 * mass[a:b], mass[a:b])
    H.ndm = ndm
    out2 = np.zeros((nh, len(STAR_FIELDS)))
    for h in range(nh):
        a, b = off[h], off[h + 1]
        member = (np.int32(b - a), index[a:b].copy(), pos[a:b].copy(), vel[a:b].copy(), mass2[a:b].copy(),
                  dens[a:b].copy())
        rec = np.zeros(1, dtype=H.halo_dtype)[0]
        rec["nmem"] = b - a
        CHP.det_mass_17(rec, member=member)
        CHP.det_center_18(rec, member=member)
        CHP.refine_centers_1b(rec, member=member)
        CHP.compute_ang_mom_19(rec, member=member)
        CHP.r_halos_1a(rec, member=member)
        CHP.det_main_axis_1b2(rec, member=member)
        CHP.det_halo_energies_1b3(rec, member=member)
        CHP.compute_spin_parameter_1c(rec)
        out2[h] = [rec[f] for f in STAR_FIELDS]
    for name in list(H.mem.keys()):
        H.deallocate(name)
    np.savez_compressed(os.path.join(HERE, "halo_case_stars.npz"), off=off, pos=pos, vel=vel, mass=mass2,
                        dens=dens, index=index.astype(np.int32), ndm=ndm, massp=0.8, out=out2,
                        fields=np.array(STAR_FIELDS), Lbox=box, Hub_pt=70.0, gravconst=430.1)
    print("halo_case_stars", nh, "halos", int(off[-1]), "members", int((index >= ndm).sum()), "stars")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HALOMAKER_REF")
    if not root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> (or set HALOMAKER_REF)")
    main(root)
