"""Record the reference's tree-brick writer and its halo-tree fields.

write_tree_brick_hdf (src/input_output.py:1048-1269) needs h5py, which is not
installed; it imports h5py inside the function, so this script puts a
recording stand-in (tests/golden/h5py_record.py) in its place and records
every group, attribute and dataset the writer creates.  Its inputs:
  * the halo/subhalo tree of the MSM fixture msm_case_2.npz (the reference's
    own select_with_MS_method_1319 output), turned into catalogue records by
    the reference's init_halos_16 (src/compute_halo_props.py:713-751);
  * seeded values for every property field the batched kernels fill (the
    writer only converts units and lays them out);
  * that fixture's member grouping (whereIam_idxs / counts, pids0_groupsorted).
Writes tests/golden/treebrick_case.npz: the inputs, the records after
init_halos_16, the header/input values, and the writer's record.

Usage (where the reference is mounted): python tests/golden/make_treebrick_golden.py /path/to/reference
"""
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PROPERTY_FIELDS = ("nmem", "ndm", "nstar", "px", "py", "pz", "vx", "vy", "vz", "Lx", "Ly", "Lz", "Lx*", "Ly*", "Lz*",
                   "sha", "shb", "shc", "m", "mdm", "m*", "r", "spin", "sigma", "sigma_dm", "sigma*", "ek", "ep",
                   "et", "rvir", "mvir", "tvir", "cvel", "rho_0", "r_c", "mcontam")
META = dict(npart=3000, nusedpart=3000, ndm=2600, nstar=400, family="all", massp=np.float64(1.0 / 3000),
            aexp=np.float64(0.8), omega_t=np.float64(0.41), age_univ=np.float64(11.2), boxsize2=np.float64(100.0),
            hubble=np.float64(0.7), mboxp=np.float64(3.9e4), numstep=7, nb_of_halos=None, nb_of_subhalos=None,
            createtime="2026-12-04 12:00:00", omega_f=0.3, omega_lambda_f=0.7, af=1.0, Lf=100.0, H_f=70.0,
            FlagPeriod=1, nMembers=20, cdm=False, method="MSM", b_init=0.2, nvoisins=32, nhop=16,
            rho_threshold=80.0, fudge=4.0, fudgepsilon=1e-5, alphap=1.0, verbose=False, megaverbose=False,
            DPMMC=False, SC=False, dcell_min=0.005, eps_SC=0.05, nsteps=1, photometry=False)


def main(refroot):
    sys.path.insert(0, HERE)
    sys.path.insert(0, os.path.join(refroot, "src"))
    import h5py_record
    sys.modules["h5py"] = h5py_record
    import halo_defs as H
    H.FORTRAN = False
    import compute_halo_props as CHP
    import input_output as IO
    d = np.load(os.path.join(HERE, "msm_case_2.npz"))
    nh, ns = int(d["nb_of_halos"]), int(d["nb_of_subhalos"])
    n = nh + ns
    H.nb_of_halos, H.nb_of_subhalos = nh, ns
    H.fsub = True
    H.numstep = META["numstep"]
    for name in ("level", "first_daughter", "mother", "first_sister"):
        H.allocate(f"{name}_1319", n, dtype=np.int32)
        H.mem[f"{name}_1319"][:] = d[name]
    H.allocate("liste_halos_o0", n + 1, dtype=H.halo_dtype)
    H.liste_halos_o0 = H.mem["liste_halos_o0"]
    CHP.init_halos_16()
    tree = H.liste_halos_o0[1:].copy()
    rng = np.random.default_rng(17)
    cat = H.liste_halos_o0
    for f in PROPERTY_FIELDS:
        if cat.dtype[f].kind == "i":
            cat[f][1:] = rng.integers(1, 5000, n)
        else:
            cat[f][1:] = rng.normal(size=n) * 10.0 ** rng.integers(-3, 4, n)
    cat["px"][1:] = rng.uniform(-55.0, 55.0, n)  # some outside [0, L): the writer wraps
    cat["mvir"][1] = np.nan  # a non-virialised one
    records = cat[1:].copy()
    H.allocate("whereIam_idxs", len(d["group_idxs"]), dtype=np.int32)
    H.allocate("whereIam_counts", len(d["group_counts"]), dtype=np.int32)
    H.mem["whereIam_idxs"][:] = d["group_idxs"]
    H.mem["whereIam_counts"][:] = d["group_counts"]
    pids0 = d["pids0_groupsorted"].astype(np.int32)
    H.allocate("pids0_groupsorted", len(pids0), dtype=np.int32)
    H.mem["pids0_groupsorted"][:] = pids0
    meta = dict(META, nb_of_halos=nh, nb_of_subhalos=ns)
    for k, v in meta.items():
        if k != "createtime":
            setattr(H, k, v)
    H.mprefix = ["", "", meta["createtime"]]
    H.mode = "full"
    H.BIG_RUN = False
    H.prefix = ""
    H.file_num = meta["numstep"]
    H.fchmod = 0o644
    H.uid, H.gid = os.getuid(), os.getgid()
    with tempfile.TemporaryDirectory() as tmp:
        H.output_dir = tmp
        IO.write_tree_brick_hdf()
    log, arrays = h5py_record.record_of(h5py_record.File.opened[-1])
    np.savez_compressed(os.path.join(HERE, "treebrick_case.npz"), level=d["level"], mother=d["mother"],
                        first_sister=d["first_sister"], first_daughter=d["first_daughter"], tree=tree,
                        records=records, member_index=H.mem["whereIam_idxs"], member_count=H.mem["whereIam_counts"],
                        pids0_groupsorted=pids0, meta=json.dumps({k: [type(v).__name__, v if not isinstance(
                            v, np.floating) else float(v)] for k, v in meta.items()}), log=json.dumps(log),
                        **{"rec_" + k: v for k, v in arrays.items()})
    for name in list(H.mem.keys()):
        H.deallocate(name)
    print("treebrick_case:", n, "structures,", len(log), "writer calls")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HALOMAKER_REF")
    if not root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> (or set HALOMAKER_REF)")
    main(root)
