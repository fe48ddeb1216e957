"""Pin the halo-property oracle against fixtures from the reference's functions.

tests/golden/halo_case.npz comes from src/compute_halo_props.py run on seeded
halos (tests/golden/make_halo_golden.py).  The oracle restates the same NumPy
formulas, so O(n) fields agree to rounding; the potential is compared where
the reference itself sums pairs (fewer than 1000 members).
"""
import os

import numpy as np

import halo_oracle

GOLD = os.path.join(os.path.dirname(__file__), "golden", "halo_case.npz")


def test_oracle_matches_reference_halo_functions():
    g = np.load(GOLD)
    f = list(g["fields"])
    ref = g["out"]
    r = halo_oracle.props(g["off"], g["pos"], g["vel"], g["mass"], g["dens"], float(g["Lbox"]), float(g["Hub_pt"]),
                          float(g["gravconst"]), nthreads=2)
    col = lambda n: ref[:, f.index(n)]
    for name in ["m", "px", "py", "pz", "vx", "vy", "vz", "r", "ek", "sigma"]:
        np.testing.assert_allclose(r[name], col(name), rtol=1e-12, atol=0, err_msg=name)
    for name in ["Lx", "Ly", "Lz"]:
        np.testing.assert_allclose(r[name], col(name), rtol=1e-10, atol=1e-12 * np.abs(col(name)).max(), err_msg=name)
    for name in ["sha", "shb", "shc"]:
        np.testing.assert_allclose(r[name], col(name), rtol=1e-10, err_msg=name)
    n = np.diff(g["off"])
    small = n < 1000
    np.testing.assert_allclose(r["ep64"][small], col("ep")[small], rtol=1e-12)
    np.testing.assert_allclose(r["spin64"][small], col("spin")[small], rtol=1e-10)


STARS = os.path.join(os.path.dirname(__file__), "golden", "halo_case_stars.npz")


def test_oracle_matches_reference_with_stars_and_cdm():
    """halo_case_stars.npz: mode 'full', H.cdm = True, stars above H.ndm and
    heavy dark-matter members -- det_mass_17's split, det_center_18's
    centre-of-mass member and sigma_dm / sigma*."""
    g = np.load(STARS)
    f = list(g["fields"])
    ref = g["out"]
    r = halo_oracle.props(g["off"], g["pos"], g["vel"], g["mass"], g["dens"], float(g["Lbox"]), float(g["Hub_pt"]),
                          float(g["gravconst"]), nthreads=2, cdm=True, index=g["index"], ndm=int(g["ndm"]),
                          massp=float(g["massp"]))
    col = lambda n: ref[:, f.index(n)]
    for name in ["ndm", "nstar"]:
        assert np.array_equal(r[name], col(name)), name
    for name in ["m", "mdm", "m*", "mcontam", "px", "py", "pz", "vx", "vy", "vz", "r", "ek", "sigma", "sigma_dm",
                 "sigma*"]:
        np.testing.assert_allclose(r[name], col(name), rtol=1e-12, atol=0, err_msg=name)
    assert (col("nstar") > 0).all() and (col("mcontam") > 0).all()
    # the centre-of-mass member differs from the densest one in most halos
    d = halo_oracle.props(g["off"], g["pos"], g["vel"], g["mass"], g["dens"], float(g["Lbox"]), float(g["Hub_pt"]),
                          float(g["gravconst"]), epot=False)
    assert np.count_nonzero(d["px"] != r["px"]) >= len(r["px"]) - 1


VIR = os.path.join(os.path.dirname(__file__), "golden", "virial_case.npz")


def test_virial_oracle_matches_reference():
    """det_vir_1b's chain (tests/golden/make_virial_golden.py) vs the restatement:
    the same NumPy/SciPy operations, so the discrete shell choices agree and the
    values agree to rounding (the direct potential enters through the oracle's
    own pair sum, 1e-12)."""
    g = np.load(VIR)
    f = list(g["fields"])
    ref = g["out"]
    r = halo_oracle.virial(g["off"], g["pos"], g["vel"], g["mass"], g["dens"], float(g["Lbox"]), float(g["Hub_pt"]),
                           float(g["gravconst"]), float(g["vir_overdens"]), float(g["rho_mean"]), int(g["nshell"]),
                           nthreads=2)
    for name in ["rvir", "mvir", "cvel", "tvir", "rho_0", "r_c", "ep", "et", "amax", "bmax", "cmax"]:
        np.testing.assert_allclose(r[name], ref[:, f.index(name)], rtol=1e-10, err_msg=name)


SC = os.path.join(os.path.dirname(__file__), "golden", "sc_case.npz")


def test_shrinking_sphere_oracle_matches_reference():
    """refine_centers_1b with SC on (tests/golden/make_sc_golden.py): the same
    centre member, and the fields about it, as the reference."""
    g = np.load(SC)
    f = list(g["fields"])
    ref = g["out"]
    r = halo_oracle.props(g["off"], g["pos"], g["vel"], g["mass"], g["dens"], float(g["Lbox"]), float(g["Hub_pt"]),
                          float(g["gravconst"]), epot=False, sc=(float(g["dcell_min"]), float(g["eps_sc"])))
    for name in ["px", "py", "pz"]:
        assert np.array_equal(r[name], ref[:, f.index(name)]), name
    for name in ["r", "sha", "shb", "shc"]:
        np.testing.assert_allclose(r[name], ref[:, f.index(name)], rtol=1e-10, err_msg=name)
    for name in ["Lx", "Ly", "Lz"]:
        col = ref[:, f.index(name)]
        np.testing.assert_allclose(r[name], col, rtol=1e-10, atol=1e-12 * np.abs(col).max(), err_msg=name)
