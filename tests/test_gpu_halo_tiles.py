"""The FP32-compensated pair kernel's tile shapes, its autotuner and the
captured launch graph of the batched halo properties.

Every tile shape (128, 256 or 512 rows per work item) must give the FP64
oracle's potential to 1e-6 relative on a catalogue that holds small halos, a
halo longer than one partner chunk (32,768 members) and a halo with coincident
members (zero separations are left out, as in the FP64 form; the fast path
meets them as a non-finite sum and recomputes the item).  The autotuner must
settle on one of the three shapes for every bucket present, and a graph
replay must give the same rows as direct launches.
"""
import os

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

import halo_oracle  # noqa: E402


@pytest.fixture(scope="module")
def cat():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from ahop_b200 import build, synthetic
    build.build()
    off, pos, vel, mass, dens = synthetic.halo_catalogue(60, seed=5, nmin=20, nmax=3000, box=100.0)
    o2, p2, v2, m2, d2 = synthetic.halo_catalogue(1, seed=6, nmin=40000, nmax=40001, box=100.0)
    n1 = off[-1]
    off = np.concatenate([off, n1 + o2[1:]])
    pos, vel, mass, dens = (np.concatenate([a, b]) for a, b in ((pos, p2), (vel, v2), (mass, m2), (dens, d2)))
    # coincident members: in halo 3 (one tile) members 5..9 sit on member 4;
    # in the large halo members 1000 and 20000 sit on member 10 (other tiles)
    a = off[3]
    pos[a + 5:a + 10] = pos[a + 4]
    b = off[-2]
    pos[b + 1000] = pos[b + 10]
    pos[b + 20000] = pos[b + 10]
    rng = np.random.default_rng(8)
    mass = mass * rng.uniform(0.5, 1.5, len(mass))
    ref = halo_oracle.epot_sums(off, pos, mass, 100.0, True, nthreads=os.cpu_count())
    return off, pos, vel, mass, dens, -430.1 * ref


def test_every_tile_shape(cat):
    from ahop_b200 import halo_props
    off, pos, vel, mass, dens, ep_ref = cat
    assert np.diff(off).max() > 32768
    try:
        for rows in (128, 256, 512):
            halo_props.set_tiles([rows] * halo_props.BUCKETS)
            g = halo_props.compute(off, pos, vel, mass, dens, 100.0, 70.0)
            np.testing.assert_allclose(g["ep64"], ep_ref, rtol=1e-12, err_msg=f"ep64, {rows} rows")
            rel = np.abs(g["ep32c"] - ep_ref) / np.abs(ep_ref)
            assert rel.max() <= 1e-6, (rows, rel.max())
            assert halo_props.tiles()["rows"] == [rows] * halo_props.BUCKETS
    finally:
        halo_props.set_tiles(None)


def test_autotuner_settles_on_a_shape(cat):
    from ahop_b200 import halo_props
    off, pos, vel, mass, dens, ep_ref = cat
    halo_props.set_tiles(None)
    assert halo_props.tiles()["rows"] == [0] * halo_props.BUCKETS
    g = halo_props.compute(off, pos, vel, mass, dens, 100.0, 70.0)
    assert halo_props.timings()["tune_ms"] > 0
    t = halo_props.tiles()
    n = np.diff(off)
    edges = [0, 512, 4096, 32768, 262144, 1 << 62]
    for b in range(halo_props.BUCKETS):
        present = bool(np.any((n >= edges[b]) & (n < edges[b + 1]) & (n > 1)))
        if present:
            assert t["rows"][b] in (128, 256, 512), t
            assert all(ms > 0 for ms in t["tune_ms"][b]), t
        else:
            assert t["rows"][b] == 0, t
    rel = np.abs(g["ep32c"] - ep_ref) / np.abs(ep_ref)
    assert rel.max() <= 1e-6
    halo_props.compute(off, pos, vel, mass, dens, 100.0, 70.0)
    assert halo_props.timings()["tune_ms"] == 0.0  # tuned once per process


def test_graph_replay_matches_direct_launches(cat):
    import torch
    from ahop_b200 import halo_props
    off, pos, vel, mass, dens, _ = cat
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    d = [t(off), t(pos), t(vel), t(mass), t(dens)]
    nh = len(off) - 1
    outs = []
    out = torch.empty((nh, halo_props.NF), dtype=torch.float64, device=dev)  # same pointer every call
    try:
        halo_props.set_tiles([256] * halo_props.BUCKETS)
        for graph in (True, True, False):
            halo_props.set_graph(graph)
            out.fill_(float("nan"))
            halo_props.compute_device(*d, out, 100.0, 70.0)
            torch.cuda.synchronize()
            outs.append((out.cpu().numpy(), halo_props.timings()["graph_replays"]))
    finally:
        halo_props.set_graph(True)
        halo_props.set_tiles(None)
    assert outs[1][1] >= 1 and outs[2][1] == -1
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][0], outs[2][0])
