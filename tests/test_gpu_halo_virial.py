"""Virial step (ahop_halo_virial) on the GPU vs the oracle and the reference.

The GPU's principal axes come from its own 3x3 eigensolver and its shell
tables are filled with atomics, so a member whose ellipsoidal radius lies
within rounding of a shell boundary may land in the neighbouring shell.  The
bar: amax/bmax/cmax and E_pot/E_tot to 1e-9 relative; rvir, mvir and the
fields derived from them to 1e-9 relative for at least 97 % of the halos and
within one shell (rvir to 2/nshell relative) for all of them.  The reference
fixture comes from src/compute_halo_props.py itself
(tests/golden/make_virial_golden.py).
"""
import os

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

import halo_oracle  # noqa: E402

VIR = os.path.join(os.path.dirname(__file__), "golden", "virial_case.npz")
DERIVED = ["rvir", "mvir", "cvel", "tvir", "rho_0", "r_c"]


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from ahop_b200 import build
    build.build()


def _gpu(off, pos, vel, mass, dens, L, hub, G, od, rho, nshell=1000):
    from ahop_b200 import halo_props
    props = halo_props.compute(off, pos, vel, mass, dens, L, hub, G)
    return halo_props.virial(off, pos, vel, mass, props, L, hub, G, od, rho, nshell=nshell)


def _compare(g, r, nshell=1000, frac=0.97):
    for name in ["amax", "bmax", "cmax", "ep", "et"]:
        np.testing.assert_allclose(g[name], r[name], rtol=1e-9, err_msg=name)
    same = np.ones(len(g["rvir"]), bool)
    for name in DERIVED:
        a, b = g[name], r[name]
        assert np.array_equal(np.isnan(a), np.isnan(b)), name
        ok = np.isnan(b) | (np.abs(a - b) <= 1e-9 * np.abs(b))
        same &= ok
    assert same.mean() >= frac, same.mean()
    fin = ~np.isnan(r["rvir"])
    assert np.all(np.abs(g["rvir"][fin] - r["rvir"][fin]) <= 2.0 / nshell * r["rvir"][fin])
    return same


def test_reference_fixture():
    d = np.load(VIR)
    f = list(d["fields"])
    g = _gpu(d["off"], d["pos"], d["vel"], d["mass"], d["dens"], float(d["Lbox"]), float(d["Hub_pt"]),
             float(d["gravconst"]), float(d["vir_overdens"]), float(d["rho_mean"]), int(d["nshell"]))
    ref = {n: d["out"][:, f.index(n)] for n in f}
    same = _compare(g, ref, frac=1.0)
    assert same.all()


def test_catalogue_vs_oracle():
    from ahop_b200 import synthetic
    off, pos, vel, mass, dens = synthetic.halo_catalogue(200, seed=91, nmin=20, nmax=20000, box=100.0)
    L, hub, G, od, rho = 100.0, 70.0, 430.1, 178.0, 2e-3
    g = _gpu(off, pos, vel, mass, dens, L, hub, G, od, rho)
    r = halo_oracle.virial(off, pos, vel, mass, dens, L, hub, G, od, rho, nthreads=os.cpu_count())
    _compare(g, r)


def test_shell_count_and_direct_limit():
    from ahop_b200 import halo_props, synthetic
    off, pos, vel, mass, dens = synthetic.halo_catalogue(40, seed=12, nmin=50, nmax=3000, box=100.0)
    props = halo_props.compute(off, pos, vel, mass, dens, 100.0, 70.0)
    g = halo_props.virial(off, pos, vel, mass, props, 100.0, 70.0, 430.1, 178.0, 2e-3, nshell=257,
                          direct_limit=500)
    r = halo_oracle.virial(off, pos, vel, mass, dens, 100.0, 70.0, 430.1, 178.0, 2e-3, nshell=257,
                           direct_limit=500, nthreads=2)
    _compare(g, r, nshell=257)
    from ahop_b200 import AhopError
    with pytest.raises(AhopError):
        halo_props.virial(off, pos, vel, mass, props, 100.0, 70.0, 430.1, 178.0, 2e-3, nshell=5000)
