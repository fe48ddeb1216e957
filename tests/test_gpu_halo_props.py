"""Batched halo properties on the GPU vs the reference fixtures and the oracle.

Tolerances: O(n) fields are FP64 reductions in a different summation order
than NumPy's, so they agree to 1e-12 relative (cross products of L to 1e-10 of
the largest component); the FP64 pair-sum potential agrees with the FP64
oracle to 1e-12; the FP32-compensated potential must be within 1e-6 relative
of the FP64 one for every halo.
"""
import os

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

import halo_oracle  # noqa: E402

GOLD = os.path.join(os.path.dirname(__file__), "golden", "halo_case.npz")


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from ahop_b200 import build
    build.build()


def _check(off, pos, vel, mass, dens, L, hub, G=430.1):
    from ahop_b200 import halo_props
    g = halo_props.compute(off, pos, vel, mass, dens, L, hub, G)
    r = halo_oracle.props(off, pos, vel, mass, dens, L, hub, G, nthreads=os.cpu_count())
    for name in ["m", "px", "py", "pz", "vx", "vy", "vz", "r", "ek", "sigma", "Ixx", "Iyy", "Izz"]:
        np.testing.assert_allclose(g[name], r[name], rtol=1e-12, err_msg=name)
    assert np.array_equal(g["icenter"], r["icenter"])
    for name in ["Lx", "Ly", "Lz", "Ixy", "Ixz", "Iyz"]:
        scale = np.maximum(np.abs(r[name]), 1e-300)
        np.testing.assert_allclose(g[name], r[name], rtol=1e-10, atol=1e-12 * scale.max(), err_msg=name)
    for name in ["sha", "shb", "shc"]:
        np.testing.assert_allclose(g[name], r[name], rtol=1e-9, err_msg=name)
    np.testing.assert_allclose(g["ep64"], r["ep64"], rtol=1e-12)
    rel32 = np.abs(g["ep32c"] - g["ep64"]) / np.abs(g["ep64"])
    assert rel32.max() <= 1e-6, rel32.max()
    np.testing.assert_allclose(g["spin64"], r["spin64"], rtol=1e-10)
    return g, r


def test_reference_fixture():
    d = np.load(GOLD)
    g, r = _check(d["off"], d["pos"], d["vel"], d["mass"], d["dens"], float(d["Lbox"]), float(d["Hub_pt"]))
    f = list(d["fields"])
    ref = d["out"]
    for name in ["m", "px", "py", "pz", "vx", "vy", "vz", "r", "ek", "sigma"]:
        np.testing.assert_allclose(g[name], ref[:, f.index(name)], rtol=1e-12, err_msg=name)
    small = np.diff(d["off"]) < 1000
    np.testing.assert_allclose(g["ep64"][small], ref[small, f.index("ep")], rtol=1e-12)


def test_catalogue_mixed_sizes():
    from ahop_b200 import synthetic
    off, pos, vel, mass, dens = synthetic.halo_catalogue(300, seed=77, nmin=20, nmax=30000, box=100.0)
    _check(off, pos, vel, mass, dens, 100.0, 70.0)


def test_tiny_halos_and_boundary():
    rng = np.random.default_rng(4)
    sizes = [1, 2, 3, 255, 256, 257, 513]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
    n = off[-1]
    pos = rng.normal(scale=0.05, size=(n, 3)) + 49.98  # straddles the +L/2 edge of a [-50, 50) box
    pos = np.mod(pos + 50.0, 100.0) - 50.0
    vel = rng.normal(size=(n, 3))
    mass = rng.uniform(0.5, 1.5, n)
    dens = rng.random(n)
    from ahop_b200 import halo_props
    g = halo_props.compute(off, pos, vel, mass, dens, 100.0, 70.0)
    r = halo_oracle.props(off, pos, vel, mass, dens, 100.0, 70.0, nthreads=2)
    np.testing.assert_allclose(g["m"], r["m"], rtol=1e-12)
    np.testing.assert_allclose(g["ep64"][1:], r["ep64"][1:], rtol=1e-12)
    assert g["ep64"][0] == 0.0 and g["ep32c"][0] == 0.0


def test_shrinking_sphere_centre():
    """refine_centers_1b with SC on: the reference's fixture exactly (same centre
    member), and a catalogue against the oracle.  The sphere's centre of mass is
    summed in another order than NumPy's, so a member within rounding of a
    sphere's surface may count on the other side; at least 95 % of the halos
    must land on the same member, and every field about the centre must then
    agree as in the default mode."""
    from ahop_b200 import halo_props, synthetic
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "sc_case.npz"))
    sc = (float(d["dcell_min"]), float(d["eps_sc"]))
    g = halo_props.compute(d["off"], d["pos"], d["vel"], d["mass"], d["dens"], float(d["Lbox"]), float(d["Hub_pt"]),
                           sc=sc)
    f = list(d["fields"])
    for name in ["px", "py", "pz"]:
        assert np.array_equal(g[name], d["out"][:, f.index(name)]), name
    np.testing.assert_allclose(g["r"], d["out"][:, f.index("r")], rtol=1e-12)
    off, pos, vel, mass, dens = synthetic.halo_catalogue(200, seed=33, nmin=20, nmax=20000, box=100.0)
    g = halo_props.compute(off, pos, vel, mass, dens, 100.0, 70.0, sc=(1e-3, 0.05))
    r = halo_oracle.props(off, pos, vel, mass, dens, 100.0, 70.0, epot=False, sc=(1e-3, 0.05))
    same = g["icenter"] == r["icenter"]
    assert same.mean() >= 0.95, same.mean()
    np.testing.assert_allclose(g["r"][same], r["r"][same], rtol=1e-12)
    with pytest.raises(Exception):
        halo_props.compute(off, pos, vel, mass, dens, 100.0, 70.0, sc=(1e-3, 0.0))


def test_stars_and_centre_of_mass():
    """Mode 'full' with stars and H.cdm: the reference's fixture
    (halo_case_stars.npz: det_mass_17's ndm, nstar, mdm, m*, mcontam;
    det_center_18's centre-of-mass member, sigma_dm, sigma*) through the host
    entry point, and a larger catalogue with stars against the oracle through
    the device entry point (member indices on the device)."""
    import torch
    from ahop_b200 import halo_props, synthetic
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", "halo_case_stars.npz"))
    kw = dict(cdm=True, index=d["index"], ndm=int(d["ndm"]), massp=float(d["massp"]))
    g = halo_props.compute(d["off"], d["pos"], d["vel"], d["mass"], d["dens"], float(d["Lbox"]), float(d["Hub_pt"]),
                           **kw)
    f = list(d["fields"])
    col = lambda n: d["out"][:, f.index(n)]
    for name in ["ndm", "nstar"]:
        assert np.array_equal(g[name], col(name)), name
    for name in ["px", "py", "pz"]:
        assert np.array_equal(g[name], col(name)), name
    for name in ["m", "mdm", "m*", "mcontam", "vx", "vy", "vz", "r", "ek", "sigma", "sigma_dm", "sigma*"]:
        np.testing.assert_allclose(g[name], col(name), rtol=1e-12, err_msg=name)
    # a catalogue with 30 % stars, device arrays
    off, pos, vel, mass, dens = synthetic.halo_catalogue(150, seed=61, nmin=20, nmax=40000, box=100.0)
    rng = np.random.default_rng(5)
    star = rng.random(len(mass)) < 0.3
    ndm = 10_000_000
    index = np.where(star, ndm + np.arange(len(mass)), np.arange(len(mass))).astype(np.int32)
    mass = np.where(star, 0.1, 1.0) * rng.uniform(0.9, 1.2, len(mass))
    r = halo_oracle.props(off, pos, vel, mass, dens, 100.0, 70.0, epot=False, cdm=True, index=index, ndm=ndm,
                          massp=1.1)
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    out = torch.zeros((len(off) - 1, halo_props.NF), dtype=torch.float64, device=dev)
    halo_props.compute_device(t(off), t(pos), t(vel), t(mass), t(dens), out, 100.0, 70.0, cdm=True,
                              d_index=t(index), ndm=ndm, massp=1.1)
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    gi = lambda n: o[:, halo_props.FIELDS.index(n)]
    for name in ["ndm", "nstar", "icenter"]:
        assert np.array_equal(gi(name), r[name]), name
    for name in ["m", "mdm", "m*", "mcontam", "px", "py", "pz", "r", "sigma", "sigma_dm", "sigma*"]:
        np.testing.assert_allclose(gi(name), r[name], rtol=1e-12, err_msg=name)
