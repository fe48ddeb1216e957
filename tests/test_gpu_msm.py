"""MSM selection and grouping on the GPU vs the restatement (pinned to the
reference) and vs the reference's own fixtures; exact integer equality."""
import glob
import os

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

import msm_oracle  # noqa: E402
import oracle  # noqa: E402

GOLD = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "msm_case_*.npz")))


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from ahop_b200 import build
    build.build()


def _run(pos, mass):
    from ahop_b200 import finder, msm
    finder.configure(mass.shape[0])
    out = finder.run(pos, mass)
    return out, msm.select()


def _check(res, ref):
    assert res["nstruct"] == ref["nstruct"]
    assert res["nb_of_halos"] == ref["nb_of_halos"] and res["nb_of_subhalos"] == ref["nb_of_subhalos"]
    assert np.array_equal(res["whereIam_parts"], ref["whereIam_parts"])
    for k in ("mother", "first_sister", "first_daughter", "level"):
        assert np.array_equal(res[k], ref[k]), k
    order, unis, idxs, counts = msm_oracle.group_members(ref["whereIam_parts"])
    assert np.array_equal(res["run_ids"], unis) and np.array_equal(res["run_counts"], counts)
    assert np.array_equal(res["run_idxs"], idxs)
    assert np.array_equal(res["pids_groupsorted"], order)  # stable grouping


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_msm_reference_fixtures(path):
    g = np.load(path)
    out, res = _run(g["pos"], g["mass"])
    assert np.array_equal(out["integer_table"], g["integer_table"])
    ref = {k: g[k] for k in ("whereIam_parts", "mother", "first_sister", "first_daughter", "level")}
    ref.update(nstruct=int(g["nstruct"]), nb_of_halos=int(g["nb_of_halos"]), nb_of_subhalos=int(g["nb_of_subhalos"]))
    _check(res, ref)


@pytest.mark.parametrize("n,nhalo,seed,nmax", [(262144, 300, 1, 20000), (60000, 60, 23, 8000)])
def test_msm_vs_oracle(n, nhalo, seed, nmax):
    from ahop_b200 import synthetic
    ps = synthetic.small_box(n, nhalo, seed=seed, nmax=nmax)
    out, res = _run(ps.pos, ps.mass)
    ref = msm_oracle.select_msm(out["real_table"], out["integer_table"], out["liste_parts"])
    _check(res, ref)
