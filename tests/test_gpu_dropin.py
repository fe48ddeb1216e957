"""The reference driver's own call sequence, replayed through the drop-in.

tests/golden/dropin_calls.npz records what src/compute_neiKDtree_mod.py
(NEI:39-124, 155-210, 738-747) passes to ``neikdtree`` with H.FORTRAN = True:
the 22 arguments of sync_from_init_adaptahop, sync_from_change_pos,
sync_others, then compute_adaptahop(np.asfortranarray(pos.T), mass) on
positions scaled by boxsize2 = 100, then close.  Replaying it through this
library's ``compute_adaptahop.neikdtree`` must give the oracle's outputs for
the same positions and parameters bit for bit; the driver's own reads
(NEI:53-60: liste_parts, density, nnodes, real_table.T, integer_table.T) are
done the same way here.
"""
import os

import numpy as np
import pytest

from conftest import gpu_available
from test_dropin_record import load_calls

pytestmark = pytest.mark.gpu


def test_reference_driver_calls_through_the_drop_in():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from ahop_b200 import build
    build.build()
    import oracle
    from compute_adaptahop import neikdtree
    calls = load_calls()
    got = None
    for name, args, _ in calls:
        if name == "close":
            # what the driver copies out before close() (NEI:53-60)
            got = dict(liste_parts=np.array(neikdtree.liste_parts[:]), density=np.array(neikdtree.density[:]),
                       nnodes=int(neikdtree.nnodes), real_table=np.array(neikdtree.real_table.T),
                       integer_table=np.array(neikdtree.integer_table.T))
        getattr(neikdtree, name)(*args)
    assert got is not None and neikdtree.density is None
    init = calls[0][1]
    change = calls[1][1]
    others = calls[2][1]
    pos, mass = calls[3][1]
    n = int(change[1])
    box = float(init[13])
    prm = oracle.default_params(n, box=box, nvoisins=int(others[8]), nhop=int(others[7]),
                                rho_threshold=float(others[4]), fudge=float(others[9]), alphap=float(others[10]),
                                nmembthresh=int(init[1]), nlevelmax=int(others[12]), nthreads=os.cpu_count())
    prm["epsilon"] = float(change[2])
    ref = oracle.run(np.ascontiguousarray(pos.T), mass, prm)
    assert got["nnodes"] == ref["nnodes"] > 0
    assert np.array_equal(got["density"], ref["density"])
    assert np.array_equal(got["liste_parts"], ref["liste_parts"])
    assert np.array_equal(got["integer_table"], ref["integer_table"])
    assert np.array_equal(got["real_table"], ref["real_table"])
