"""One snapshot through the device pipeline (finder, MSM selection, member
gather, batched properties) against the same steps through the host entry
points: the reference's grouping (NumPy argsort/unique of whereIam_parts,
NEI:107-119) and gather (CHP:497-506) on the host, then ahop_halo_props on
host buffers.  Same kernels on the same members in the same order, so every
property row must agree bit for bit."""
import os

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from ahop_b200 import build
    build.build()


def test_device_pipeline_matches_host_steps():
    from ahop_b200 import finder, halo_props, msm, pipeline, synthetic
    ps = synthetic.small_box(120_000, 120, seed=31, nmax=8000)
    halo_props.set_tiles([256] * halo_props.BUCKETS)
    try:
        res = pipeline.run_snapshot(ps.pos, ps.vel, ps.mass, box=1.0, hub=70.0, epot=3, particle_views=True)
        finder.configure(ps.n)
        out = finder.run(ps.pos, ps.mass)
        sel = msm.select()
        assert np.array_equal(sel["whereIam_parts"], res["whereIam_parts"])
        w = sel["whereIam_parts"]
        order = np.argsort(w, kind="stable")
        ids, idxs, counts = np.unique(w[order], return_index=True, return_counts=True)
        keep = ids > 0
        ids, idxs, counts = ids[keep], idxs[keep], counts[keep]
        assert np.array_equal(res["ids"], ids)
        members = np.concatenate([order[i:i + c] for i, c in zip(idxs, counts)])
        off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        assert np.array_equal(res["offsets"], off)
        g = halo_props.compute(off, ps.pos[members], ps.vel[members], ps.mass[members], out["density"][members],
                               1.0, 70.0, epot=3)
        host = np.stack([g[f] for f in halo_props.FIELDS], 1)
        assert res["props"].shape == host.shape
        assert np.array_equal(res["props"], host, equal_nan=True)
    finally:
        halo_props.set_tiles(None)


def test_pipeline_with_stars_centre_of_mass_and_virial_step():
    """A box with 15 % stars (dark matter first, ndm), the centre-of-mass
    centre and the virial step inside the snapshot pipeline, against the host
    entry points on the host-gathered members with their particle indices:
    every property row bit for bit; the virial rows to 1e-9 (the virial
    step's shell sums are shared-memory atomics, so their last bits depend on
    the order in which members land)."""
    from ahop_b200 import finder, halo_props, msm, pipeline, synthetic
    ps = synthetic.clustered_box(100_000, 100, seed=37, nmax=8000, star_fraction=0.15)
    assert ps.ndm is not None and 0 < ps.ndm < ps.n
    halo_props.set_tiles([256] * halo_props.BUCKETS)
    try:
        kw = dict(ndm=ps.ndm, cdm=True, massp=1.5 / ps.n)
        res = pipeline.run_snapshot(ps.pos, ps.vel, ps.mass, box=1.0, hub=70.0, epot=3, particle_views=True,
                                    vir_overdens=178.0, rho_mean=1.0, **kw)
        finder.configure(ps.n)
        out = finder.run(ps.pos, ps.mass)
        sel = msm.select()
        w = sel["whereIam_parts"]
        order = np.argsort(w, kind="stable")
        ids, idxs, counts = np.unique(w[order], return_index=True, return_counts=True)
        keep = ids > 0
        idxs, counts = idxs[keep], counts[keep]
        members = np.concatenate([order[i:i + c] for i, c in zip(idxs, counts)])
        off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        g = halo_props.compute(off, ps.pos[members], ps.vel[members], ps.mass[members], out["density"][members],
                               1.0, 70.0, epot=3, index=members.astype(np.int32), **kw)
        host = np.stack([g[f] for f in halo_props.FIELDS], 1)
        assert np.array_equal(res["props"], host, equal_nan=True)
        assert g["nstar"].sum() > 0 and np.array_equal(g["ndm"] + g["nstar"], np.diff(off).astype(float))
        v = halo_props.virial(off, ps.pos[members], ps.vel[members], ps.mass[members], g, 1.0, 70.0, 430.1, 178.0,
                              1.0, ep="ep64")
        vh = np.stack([v[f] for f in halo_props.VIR_FIELDS], 1)
        assert res["virial"].shape == vh.shape
        assert np.array_equal(np.isnan(res["virial"]), np.isnan(vh))
        np.testing.assert_allclose(res["virial"], vh, rtol=1e-9, equal_nan=True)
        assert np.isfinite(res["virial"][:, 0]).mean() > 0.5
    finally:
        halo_props.set_tiles(None)


def test_tree_brick_from_the_pipeline(tmp_path):
    """The tree-brick catalogue of a pipeline run (ahop_b200.tree_bricks),
    written through the recording h5py stand-in: one record per structure,
    property fields equal to the pipeline's rows after the reference's unit
    conversion, the tree fields from the selection, members as grouped."""
    import json
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import h5py_record
    from ahop_b200 import halo_props, pipeline, synthetic, tree_bricks as T
    ps = synthetic.clustered_box(60_000, 60, seed=41, nmax=6000, star_fraction=0.15)
    res = pipeline.run_snapshot(ps.pos * 100.0, ps.vel, ps.mass, box=100.0, hub=70.0, epot=3, particle_views=True,
                                ndm=ps.ndm, rho_mean=1.0)
    cat, idx, cnt, pids = T.from_snapshot(res, numstep=3)
    assert len(cat) == res["nstruct"] and np.array_equal(cat["id"], np.arange(1, len(cat) + 1))
    k = res["ids"] - 1
    F = lambda f: res["props"][:, halo_props.FIELDS.index(f)]
    assert np.array_equal(cat["nmem"][k], np.diff(res["offsets"]))
    assert np.array_equal(cat["nstar"][k], F("nstar").astype(np.int32))
    np.testing.assert_array_equal(cat["m"][k], F("m"))
    assert cnt.sum() == ps.n and np.array_equal(np.sort(pids), np.arange(ps.n))
    meta = dict(npart=ps.n, nusedpart=ps.n, ndm=ps.ndm, nstar=ps.n - ps.ndm, family="all", massp=1.0 / ps.n,
                aexp=1.0, omega_t=0.3, age_univ=13.7, boxsize2=100.0, hubble=0.7, mboxp=1.0, numstep=3,
                nb_of_halos=res["nb_of_halos"], nb_of_subhalos=res["nb_of_subhalos"], createtime="now",
                omega_f=0.3, omega_lambda_f=0.7, af=1.0, Lf=100.0, H_f=70.0, FlagPeriod=1, nMembers=20, cdm=False,
                method="MSM", b_init=0.2, nvoisins=32, nhop=16, rho_threshold=80.0, fudge=4.0, fudgepsilon=1e-5,
                alphap=1.0, verbose=False, megaverbose=False, DPMMC=False, SC=False, dcell_min=0.005, eps_SC=0.05,
                nsteps=1, photometry=False)
    f = h5py_record.File(str(tmp_path / "tb.h5"), "w")
    T.write(f, meta, cat, idx, cnt, pids)
    log, arrays = h5py_record.record_of(f)
    halo = [e for e in log if e["op"] == "dataset" and e["path"] == "/catalog/halo"][0]
    written = arrays[halo["data"]]
    np.testing.assert_array_equal(written["m"][k], F("m") * 1e11)
    np.testing.assert_array_equal(written["px"][k], np.mod(F("px") / 100.0, 1.0))
    assert json.loads([e for e in log if e.get("name") == "field_units"][0]["value"]["v"])["m"] == "Msun"
