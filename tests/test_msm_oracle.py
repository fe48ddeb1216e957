"""Pin the MSM restatement against fixtures made by the reference's own
select_with_MS_method_1319 and member grouping (tests/golden/make_msm_golden.py)."""
import glob
import os

import numpy as np
import pytest

import msm_oracle

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "msm_case_*.npz")))


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_msm_matches_reference(path):
    g = np.load(path)
    r = msm_oracle.select_msm(g["real_table"], g["integer_table"], g["liste_parts"])
    assert r["nstruct"] == int(g["nstruct"])
    assert r["nb_of_halos"] == int(g["nb_of_halos"])
    assert r["nb_of_subhalos"] == int(g["nb_of_subhalos"])
    assert np.array_equal(r["whereIam_parts"], g["whereIam_parts"])
    for k in ("mother", "first_sister", "first_daughter", "level"):
        assert np.array_equal(r[k], g[k]), k
    order, unis, idxs, counts = msm_oracle.group_members(r["whereIam_parts"])
    assert np.array_equal(unis, g["group_unis"]) and np.array_equal(counts, g["group_counts"])
    assert np.array_equal(idxs, g["group_idxs"])
    # members per structure agree as sets (numpy's default argsort is not stable)
    ref = g["pids0_groupsorted"]
    for a, c in zip(idxs, counts):
        assert np.array_equal(np.sort(order[a:a + c]), np.sort(ref[a:a + c]))


def test_msm_golden_present():
    assert len(GOLD) >= 3
