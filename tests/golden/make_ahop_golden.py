"""Generate AdaptaHOP golden fixtures by running the REFERENCE's own finder.

The reference ships no tests or fixtures, and its Fortran module cannot be
compiled here (no Fortran compiler).  Its pure-Python finder
(src/compute_neiKDtree_mod.py, ``H.FORTRAN = False``, ``H.SCIPY = False``) is
importable, so this script runs it on small seeded particle sets and commits
its outputs as fixtures.  They pin the CPU oracle (a restatement of
fortran/compute_adaptahop.f90) before the oracle is trusted as the checker of
the CUDA path.

Known differences between that Python path and the Fortran, handled here or in
the comparison (tests/test_oracle_golden.py):
  * ``H.pi`` is numpy's pi; the Fortran's ``pi`` is the single-precision
    literal 3.141592654 promoted to real(8) (f90:58).  The script sets
    ``H.pi`` to the Fortran value before running, so density matches to
    summation-order rounding (numpy pairwise sums, ``/r`` instead of ``*1/r``).
  * The Python path does not renumber nodes (f90:987-1131), so nodes are
    compared as sets and memberships through the induced node-id map.
  * treat_particles_new_13141 wraps with the opposite sign and picks posref
    from the last member (src/compute_neiKDtree_mod.py:1210,1218): node
    positions/radii only agree for halos that do not straddle the periodic
    boundary; the fixtures record which nodes do.

Usage (in the development container, where the reference is mounted):
    python tests/golden/make_ahop_golden.py /path/to/reference
Writes tests/golden/ahop_case*.npz.
"""
import os
import sys
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))

CASES = [
    # name, npart, nhalo, seed, nmax
    ("ahop_case_a", 3000, 8, 11, 600),
    ("ahop_case_b", 5000, 16, 12, 800),
    ("ahop_case_c", 4000, 3, 13, 1500),
    # a larger box: halos of up to 12,000 particles with subhalos, so the
    # structure tree has several levels of significance tests
    ("ahop_case_d", 40000, 30, 15, 12000),
]


def run_case(H, NEI, pos, mass):
    n = mass.shape[0]
    H.nbPes = 1
    H.npart = n
    H.nusedpart = n
    H.nvoisins = 32
    H.nhop = 16
    H.rho_threshold = 80.0
    H.fudge = 4.0
    H.fudgepsilon = 1e-5
    H.alphap = 1.0
    H.nMembers = 20
    H.nmembthresh = 20
    H.nlevelmax = 30
    H.method = "MSM"
    H.Lf = 1.0
    H.boxsize2 = 1.0
    H.xlong = H.ylong = H.zlong = 1.0
    H.boxarr = np.array([1.0, 1.0, 1.0])
    H.xlongs2 = H.ylongs2 = H.zlongs2 = 0.5
    H.pi = np.float64(np.float32(3.141592654))
    H.allocate("pos_10", (n, 3), np.float64)
    H.mem["pos_10"][:] = pos
    H.allocate("mass_10", n, np.float64)
    H.mem["mass_10"][:] = mass
    H.allocate("whereIam_parts", n, np.int32)
    NEI.init_group_members()  # module-level membership cache (src/compute_neiKDtree_mod.py:733)
    NEI.change_pos_1310()
    NEI.create_tree_structure_1311()
    NEI.compute_mean_density_and_np_1312()
    NEI.find_local_maxima_1313()
    out = {}
    out["density"] = H.mem["density_1312"].copy()
    out["iparneigh"] = H.mem["iparneigh_1312"][: H.nhop].T.copy()  # (n, nhop) 1-based
    out["group"] = H.mem["igrouppart_1313"].copy()
    out["ngroups"] = np.int32(H.ngroups)
    orig = NEI.compute_saddle_list_13140
    snap = {}

    def wrapped():
        orig()
        off = [0]
        isad, rho = [], []
        for g in H.group:
            k = int(g.nhnei)
            if k > 0:
                isad.extend(int(x) for x in g.isad_gr[:k])
                rho.extend(float(x) for x in g.rho_saddle_gr[:k])
            off.append(len(isad))
        snap["saddle_offsets"] = np.array(off, np.int32)
        snap["saddle_isad"] = np.array(isad, np.int32)
        snap["saddle_rho"] = np.array(rho, np.float64)

    NEI.compute_saddle_list_13140 = wrapped
    try:
        NEI.create_group_tree_1314()
    finally:
        NEI.compute_saddle_list_13140 = orig
    out.update(snap)
    nn = int(H.nnodes)
    nodes = H.node_0[1:nn + 1]
    out["node_real"] = np.stack([nodes[f] for f in ("rho_saddle", "density", "densmax", "radius", "truemass",
                                                    "px", "py", "pz")], axis=1).astype(np.float64)
    out["node_int"] = np.stack([nodes[f] for f in ("mass", "level", "mother", "firstchild", "nsisters",
                                                   "sister")], axis=1).astype(np.int32)
    out["whereIam_parts"] = H.mem["whereIam_parts"].copy()
    out["nnodes"] = np.int32(nn)
    for name in list(H.mem.keys()):
        H.deallocate(name)
    return out


def main(refroot):
    sys.path.insert(0, os.path.join(refroot, "src"))
    sys.path.insert(0, os.path.join(REPO, "halomaker-python_b200"))
    import halo_defs as H
    H.FORTRAN = False
    H.SCIPY = False
    H.verbose = False
    H.megaverbose = False
    import compute_neiKDtree_mod as NEI
    from ahop_b200 import synthetic
    for name, npart, nhalo, seed, nmax in CASES:
        ps = synthetic.small_box(npart, nhalo, seed=seed, nmax=nmax)
        out = run_case(H, NEI, ps.pos, ps.mass)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), pos=ps.pos, mass=ps.mass, **out)
        print(name, "ngroups", int(out["ngroups"]), "nnodes", int(out["nnodes"]))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HALOMAKER_REF")
    if not root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> (or set HALOMAKER_REF)")
    main(root)
