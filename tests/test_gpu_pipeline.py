"""One snapshot through the device pipeline (finder, MSM selection, member
gather, batched properties) against the same steps through the host entry
points: the reference's grouping (NumPy argsort/unique of whereIam_parts,
NEI:107-119) and gather (CHP:497-506) on the host, then ahop_halo_props on
host buffers.  Same kernels on the same members in the same order, so every
property row must agree bit for bit."""
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
