"""Golden fixtures for the RAMSES particle reader, from the REFERENCE itself.

Writes the synthetic part files of ramses_files.CASES into a temporary
directory and reads them with the reference's own per-file reader
_read_ramses_new_1010 (src/input_output.py:624-760), driven the way
read_ramses_new_101 drives it (src/input_output.py:856-989: a counting pass
over all files, then the dense arrays sized from it and a loading pass), for
family = all, dm and star, with the stellar payload off.  Stores pos_10,
vel_10, mass_10 (and source_pid_10 for a single family) with the counts in
tests/golden/ramses_<case>_<family>.npz.

Usage (where the reference is mounted):
    python tests/golden/make_ramses_golden.py /path/to/reference
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_with_reference(IO, H, outdir, version, family):
    kwargs = {"repository": outdir, "rver": f"Ra{version}", "nchar": "00001", "ndim": 3,
              "scale_l": ramses_files.SCALE_L, "scale_t": ramses_files.SCALE_T, "snapshot_age": 0.0,
              "count_only": True, "family": family, "stellar_payload": False, "m0_skip": None,
              "stellar_descriptor": {"m0_skip": None, "chem_indices": {}, "nchem": 0}}
    H.family = family
    H.stellar_payload = False
    ncpu = len([f for f in os.listdir(outdir) if f.startswith("part_")])
    ndm = nstar = nsel = 0
    for icpu in range(1, ncpu + 1):
        a, b, c = IO._read_ramses_new_1010(icpu, kwargs)
        ndm += a
        nstar += b
        nsel += c
    H.ndm = ndm if family in {"all", "dm"} else 0
    for name in ("pos_10", "vel_10", "mass_10", "source_pid_10"):
        if H.allocated(name):
            H.deallocate(name)
    H.allocate("pos_10", (nsel, 3), dtype=np.float64)
    H.allocate("vel_10", (nsel, 3), dtype=np.float64)
    H.allocate("mass_10", (nsel,), dtype=np.float64)
    if family != "all":
        H.allocate("source_pid_10", (nsel,), dtype=np.int64)
        H.mem["source_pid_10"][:] = -1
    kwargs.update(count_only=False, ndm=H.ndm, nselected=nsel)
    for icpu in range(1, ncpu + 1):
        IO._read_ramses_new_1010(icpu, kwargs)
    out = dict(pos=H.mem["pos_10"].copy(), vel=H.mem["vel_10"].copy(), mass=H.mem["mass_10"].copy(),
               ndm=ndm, nstar=nstar, nselected=nsel)
    if family != "all":
        out["source_pid"] = H.mem["source_pid_10"].copy()
    for name in ("pos_10", "vel_10", "mass_10", "source_pid_10"):
        if H.allocated(name):
            H.deallocate(name)
    return out


def main(refroot):
    sys.path.insert(0, os.path.join(refroot, "src"))
    import halo_defs as H
    H.verbose = False
    H.megaverbose = False
    H.nbPes = 1
    import input_output as IO
    for case in ramses_files.CASES:
        with tempfile.TemporaryDirectory() as tmp:
            paths = ramses_files.write_case(tmp, case["seed"], case["version"], case["ncpu"], case["ndm"],
                                            case["nstar"], case["nother"])
            outdir = os.path.dirname(paths[0])
            for family in ("all", "dm", "star"):
                if family == "star" and case["nstar"] == 0:
                    continue
                r = read_with_reference(IO, H, outdir, case["version"], family)
                dst = os.path.join(HERE, f"ramses_{case['name']}_{family}.npz")
                np.savez_compressed(dst, **r, **{"w_" + k: v for k, v in case.items() if k != "name"}, family=family,
                                    scale_l=ramses_files.SCALE_L, scale_t=ramses_files.SCALE_T)
                print(dst, r["ndm"], r["nstar"], r["nselected"])


sys.path.insert(0, HERE)
import ramses_files  # noqa: E402

if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HALOMAKER_REF")
    if not root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> (or set HALOMAKER_REF)")
    main(root)
