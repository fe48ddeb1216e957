"""Record how the reference's own driver calls the f2py module.

The drop-in boundary is the f2py object ``compute_adaptahop.neikdtree``.  This
script imports the reference's driver, src/compute_neiKDtree_mod.py, with
``H.FORTRAN = True`` and a recording stand-in for the f2py extension first on
``sys.path``, then runs the driver's own init_adaptahop_130 (NEI:155-197) and
compute_adaptahop_131 (NEI:39-124: change_pos_1310, sync_fortran,
compute_adaptahop, the reads of the module arrays, close, the MSM selection)
on the ahop_case_a golden box in a 100-unit box (so the unit scale of
change_pos_1310, NEI:205, is exercised).

The stand-in records every call on ``neikdtree``: the subroutine name, every
argument's Python type and value, and for arrays their dtype, shape and
memory order (the driver passes np.asfortranarray(pos.T)).  It answers
compute_adaptahop with the golden box's outputs of the reference's Python
finder (scaled positions do not change them: AdaptaHOP is scale-free in
density rank and topology), so the driver proceeds through its selection.
The record is written to tests/golden/dropin_calls.npz: the call list as JSON
and the array arguments by call and position.

Usage (where the reference is mounted): python tests/golden/make_dropin_golden.py /path/to/reference
"""
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BOX = 100.0


class Recorder:
    """Stand-in for the f2py module object: records calls, serves outputs."""

    def __init__(self, golden):
        self.calls = []
        self.arrays = {}
        self.golden = golden
        self.liste_parts = self.density = self.real_table = self.integer_table = None
        self.nnodes = 0

    def _record(self, name, args):
        k = len(self.calls)
        rec = []
        for j, a in enumerate(args):
            if isinstance(a, np.ndarray):
                key = f"c{k}_a{j}"
                self.arrays[key] = np.array(a, copy=True, order="K")
                rec.append({"type": "ndarray", "key": key, "dtype": str(a.dtype), "shape": list(a.shape),
                            "f_contiguous": bool(a.flags.f_contiguous), "c_contiguous": bool(a.flags.c_contiguous)})
            elif isinstance(a, (bool, np.bool_)):
                rec.append({"type": type(a).__name__, "value": bool(a)})
            elif isinstance(a, (int, np.integer)):
                rec.append({"type": type(a).__name__, "value": int(a)})
            elif isinstance(a, (float, np.floating)):
                rec.append({"type": type(a).__name__, "value": float(a)})
            elif isinstance(a, str):
                rec.append({"type": "str", "value": a})
            else:
                raise TypeError(f"{name} argument {j}: {type(a)}")
        self.calls.append({"name": name, "args": rec})

    def sync_from_init_adaptahop(self, *args):
        self._record("sync_from_init_adaptahop", args)

    def sync_from_change_pos(self, *args):
        self._record("sync_from_change_pos", args)

    def sync_others(self, *args):
        self._record("sync_others", args)

    def compute_adaptahop(self, *args):
        self._record("compute_adaptahop", args)
        g = self.golden
        self.liste_parts = g["whereIam_parts"].astype(np.int32)
        self.density = g["density"].astype(np.float64)
        self.nnodes = np.int32(g["nnodes"])
        self.real_table = np.asfortranarray(g["node_real"].T)
        self.integer_table = np.asfortranarray(g["node_int"].T)

    def close(self):
        self._record("close", ())
        self.liste_parts = self.density = self.real_table = self.integer_table = None


def main(refroot):
    golden = np.load(os.path.join(HERE, "ahop_case_a.npz"))
    rec = Recorder(golden)
    stub = types.ModuleType("compute_adaptahop")
    stub.neikdtree = rec
    sys.modules["compute_adaptahop"] = stub
    sys.path.insert(0, os.path.join(refroot, "src"))
    import halo_defs as H
    H.FORTRAN = True
    H.SCIPY = False
    H.verbose = False
    H.megaverbose = False
    import compute_neiKDtree_mod as NEI
    pos, mass = golden["pos"], golden["mass"]
    n = mass.shape[0]
    # the snapshot's cosmology and the finder parameters (HaloMaker defaults)
    H.npart = n
    H.nusedpart = n
    H.nbPes = 4
    H.Lf = BOX
    H.H_f = 70.0
    H.omega_f = 0.3
    H.omega_lambda_f = 0.7
    H.af = 1.0
    H.aexp = 1.0
    H.nMembers = 20
    H.nvoisins = 32
    H.nhop = 16
    H.rho_threshold = 80.0
    H.fudge = 4.0
    H.fudgepsilon = 1e-5
    H.alphap = 1.0
    H.nlevelmax = 30
    H.method = "MSM"
    H.optimize_nodes = False
    H.massp = np.float64(1.0 / n)
    H.boxsize = BOX
    H.allocate("pos_10", (n, 3), np.float64)
    H.mem["pos_10"][:] = pos  # [-0.5, 0.5): the frame the reader leaves (input_output.py:511)
    H.allocate("mass_10", n, np.float64)
    H.mem["mass_10"][:] = mass
    H.allocate("whereIam_parts", n, np.int32)
    NEI.init_adaptahop_130()
    NEI.compute_adaptahop_131()
    np.savez_compressed(os.path.join(HERE, "dropin_calls.npz"), calls=json.dumps(rec.calls), **rec.arrays)
    print("dropin_calls:", [c["name"] for c in rec.calls], "nb_of_halos", int(H.nb_of_halos))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HALOMAKER_REF")
    if not root:
        sys.exit(f"usage: python {os.path.basename(__file__)} <reference checkout> (or set HALOMAKER_REF)")
    main(root)
