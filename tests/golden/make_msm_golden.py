"""Golden fixtures for the MSM halo/subhalo selection, from the REFERENCE itself.

Feeds the finder outputs (node tables and membership) of the AdaptaHOP golden
boxes, as computed by the CPU oracle, to the reference's
select_with_MS_method_1319 (src/compute_neiKDtree_mod.py:260-464) and to its
member grouping (NEI:107-119), and stores the results in
tests/golden/msm_case*.npz.

Usage (where the reference is mounted): python tests/golden/make_msm_golden.py /path/to/reference
"""
import glob
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def main(refroot):
    sys.path.insert(0, os.path.join(refroot, "src"))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    sys.path.insert(0, os.path.join(REPO, "halomaker-python_b200"))
    import halo_defs as H
    H.FORTRAN = False
    H.verbose = False
    H.megaverbose = False
    import compute_neiKDtree_mod as NEI
    import oracle
    from ahop_b200 import synthetic

    cases = [(p, dict(np.load(p))) for p in sorted(glob.glob(os.path.join(HERE, "ahop_case*.npz")))]
    # plus a larger box with deeper trees
    ps = synthetic.small_box(100000, 100, seed=8, nmax=20000)
    cases.append(("msm_big", {"pos": ps.pos, "mass": ps.mass}))
    for k, (name, g) in enumerate(cases):
        n = g["mass"].shape[0]
        r = oracle.run(g["pos"], g["mass"], oracle.default_params(n, nthreads=4))
        nn = r["nnodes"]
        H.nnodes = nn
        H.nusedpart = n
        H.npart = n
        H.node_0 = np.zeros(nn + 1, dtype=H.node_dtype)
        rt, it = r["real_table"], r["integer_table"]
        for j, f in enumerate(("rho_saddle", "density", "densmax", "radius", "truemass", "px", "py", "pz")):
            H.node_0[f][1:] = rt[:, j]
        for j, f in enumerate(("mass", "level", "mother", "firstchild", "nsisters", "sister")):
            H.node_0[f][1:] = it[:, j]
        H.allocate("whereIam_parts", n, np.int32)
        H.mem["whereIam_parts"][:] = r["liste_parts"]
        if not (it[:, 3] > 0).any():
            # the reference indexes an empty array here (NEI:267-268) and raises
            print(name, "skipped: no node has children")
            for nm in list(H.mem.keys()):
                H.deallocate(nm)
            continue
        NEI.select_with_MS_method_1319()
        wp = H.mem["whereIam_parts"].copy()
        out = dict(pos=g["pos"], mass=g["mass"], real_table=rt, integer_table=it, liste_parts=r["liste_parts"],
                   whereIam_parts=wp, nstruct=np.int32(H.nstruct), nb_of_halos=np.int32(H.nb_of_halos),
                   nb_of_subhalos=np.int32(H.nb_of_subhalos),
                   mother=H.mem["mother_1319"].copy(), first_sister=H.mem["first_sister_1319"].copy(),
                   first_daughter=H.mem["first_daughter_1319"].copy(), level=H.mem["level_1319"].copy())
        # member grouping (NEI:107-119)
        argsort = np.argsort(wp)
        unis, idxs, counts = np.unique(wp[argsort], return_index=True, return_counts=True)
        out.update(pids0_groupsorted=np.arange(n)[argsort], group_unis=unis, group_idxs=idxs,
                   group_counts=counts)
        for nm in list(H.mem.keys()):
            H.deallocate(nm)
        fn = os.path.join(HERE, f"msm_case_{k}.npz")
        np.savez_compressed(fn, **out)
        print(fn, "nnodes", nn, "nstruct", int(out["nstruct"]), "halos", int(out["nb_of_halos"]))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HALOMAKER_REF")
    if not root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> (or set HALOMAKER_REF)")
    main(root)
