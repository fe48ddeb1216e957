"""Seeded synthetic particle sets standing in for RAMSES snapshots.

No simulation snapshot is available, so every workload is drawn from a seeded
NumPy PCG64 generator with the shapes and value distributions of the
reference's target boxes: NFW halos (concentration 10, virial radius
``0.01 * (n/1000)**(1/3)`` box units) holding 0-4 NFW subhalos of 2-10 % of
the host's count placed 0.3-0.8 r_vir from the centre, plus a uniform
background.  Positions are returned in ``[-L/2, L/2)`` -- the frame the
reference hands to its finder after ``change_pos_1310``
(src/compute_neiKDtree_mod.py:200-210, src/input_output.py:511) -- as a
``(N, 3)`` float64 array; masses are float64.

Halo particle counts follow dN/dn ~ n**slope on [nmin, nmax]; when the caller
asks for a fixed halo fraction of the particles, the drawn counts are scaled
by one common factor (shape preserved) so that their sum matches it.
"""
from __future__ import annotations

import dataclasses
import numpy as np

_NFW_C = 10.0


@dataclasses.dataclass
class ParticleSet:
    pos: np.ndarray           # (N, 3) float64 in [-L/2, L/2)
    vel: np.ndarray           # (N, 3) float64
    mass: np.ndarray          # (N,)  float64
    halo_id: np.ndarray       # (N,)  int32, -1 for background particles
    halo_counts: np.ndarray   # (nhalo,) int64 particles per host halo (incl. subhalos)
    box: float = 1.0
    seed: int = 0
    ndm: int | None = None    # particles [0, ndm) are dark matter, the rest stars (None: all dark matter)

    @property
    def n(self) -> int:
        return int(self.mass.shape[0])


def _powerlaw_counts(rng, nhalo, slope, nmin, nmax):
    a = slope + 1.0
    u = rng.random(nhalo)
    lo, hi = nmin ** a, nmax ** a
    return np.floor((lo + u * (hi - lo)) ** (1.0 / a)).astype(np.int64)


_NFW_TABLE = None


def _nfw_radius(rng, n, rvir, c=_NFW_C):
    """Radii r = x*rvir with x from the NFW enclosed-mass inverse CDF on [0,1]."""
    global _NFW_TABLE
    if _NFW_TABLE is None:
        x = np.linspace(0.0, 1.0, 4097)
        m = np.log1p(c * x) - c * x / (1.0 + c * x)
        _NFW_TABLE = (m / m[-1], x)
    cdf, x = _NFW_TABLE
    return np.interp(rng.random(n), cdf, x) * rvir


def _isotropic(rng, n):
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True) + 1e-300
    return v


def _nfw_blob(rng, n, centre, rvir):
    r = _nfw_radius(rng, n, rvir)
    return centre[None, :] + r[:, None] * _isotropic(rng, n)


def clustered_box(npart: int, nhalo: int, seed: int, halo_fraction: float = 0.6,
                  nmin: int = 20, nmax: int = 20000, slope: float = -1.9,
                  box: float = 1.0, star_fraction: float = 0.0,
                  sigma_v0: float = 100.0, sigma_bulk: float = 300.0) -> ParticleSet:
    """Clustered periodic box: NFW halos with subhalos plus a uniform background.

    ``star_fraction`` > 0 turns that fraction of each halo's particles into
    stars of mass 0.1 m concentrated in the halo core (half-mass radius 0.05
    r_vir); masses are then renormalised to a total of 1, and the particles
    are ordered dark matter first, then stars (as the RAMSES reader lays out
    family 'all'), with ``ndm`` the dark-matter count.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = _powerlaw_counts(rng, nhalo, slope, nmin, nmax)
    target = int(round(halo_fraction * npart))
    if counts.sum() > 0 and target > 0:
        counts = np.maximum(nmin, np.floor(counts * (target / counts.sum()))).astype(np.int64)
        diff = target - int(counts.sum())
        counts[np.argmax(counts)] += diff
    nhalo_tot = int(counts.sum())
    if nhalo_tot > npart:
        raise ValueError("halo particles exceed npart")
    pos = np.empty((npart, 3), np.float64)
    vel = np.empty((npart, 3), np.float64)
    hid = np.full(npart, -1, np.int32)
    is_star = np.zeros(npart, bool)
    off = 0
    for ih, n in enumerate(counts):
        n = int(n)
        centre = rng.random(3) * box
        rvir = 0.01 * box * (n / 1000.0) ** (1.0 / 3.0)
        nsub = int(rng.integers(0, 5))
        sub_n = []
        left = n
        for _ in range(nsub):
            k = int(n * rng.uniform(0.02, 0.10))
            if k < 2 or k >= left - 2:
                continue
            sub_n.append(k)
            left -= k
        p = [_nfw_blob(rng, left, centre, rvir)]
        for k in sub_n:
            d = rng.uniform(0.3, 0.8) * rvir
            sc = centre + d * _isotropic(rng, 1)[0]
            p.append(_nfw_blob(rng, k, sc, 0.01 * box * (k / 1000.0) ** (1.0 / 3.0)))
        blob = np.concatenate(p, axis=0)
        sig = sigma_v0 * (n / 1000.0) ** (1.0 / 3.0)
        v = rng.normal(scale=sig, size=(n, 3)) + rng.normal(scale=sigma_bulk, size=3)[None, :]
        if star_fraction > 0.0:
            ns = int(round(star_fraction * n))
            if ns > 0:
                # stars: Plummer-like core with half-mass radius 0.05 rvir
                a = 0.05 * rvir / 1.305
                u = rng.random(ns)
                rs = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
                rs = np.minimum(rs, rvir)
                blob[:ns] = centre[None, :] + rs[:, None] * _isotropic(rng, ns)
                is_star[off:off + ns] = True
        pos[off:off + n] = blob
        vel[off:off + n] = v
        hid[off:off + n] = ih
        off += n
    nu = npart - off
    pos[off:] = rng.random((nu, 3)) * box
    vel[off:] = rng.normal(scale=sigma_v0 * 0.3, size=(nu, 3))
    # periodic wrap to [0, L) then shift to [-L/2, L/2)
    pos = np.mod(pos, box)
    pos[pos >= box] = 0.0
    pos -= 0.5 * box
    # the shift can round x + (-0.5) up to exactly +0.5; keep the half-open range
    pos[pos >= 0.5 * box] = -0.5 * box
    # shuffle so particle index carries no halo structure (as in a snapshot)
    perm = rng.permutation(npart)
    pos, vel, hid, is_star = pos[perm], vel[perm], hid[perm], is_star[perm]
    mass = np.full(npart, 1.0 / npart, np.float64)
    ndm = None
    if star_fraction > 0.0:
        mass[is_star] *= 0.1
        mass /= mass.sum()
        order = np.argsort(is_star, kind="stable")  # dark matter first
        pos, vel, hid, mass = pos[order], vel[order], hid[order], mass[order]
        ndm = int(npart - np.count_nonzero(is_star))
    return ParticleSet(np.ascontiguousarray(pos), np.ascontiguousarray(vel), mass, hid, counts, box, seed, ndm)


# Named workloads (seeds fixed per workload).
def workload(name: str) -> ParticleSet:
    if name == "c1_262k":
        return clustered_box(262_144, 300, seed=1, nmax=20_000)
    if name == "c2_256cubed":
        return clustered_box(16_777_216, 19_200, seed=2, nmax=2_000_000)
    if name == "c4_2m":
        return clustered_box(2_097_152, 2_000, seed=4, nmax=50_000)
    if name == "c5_512cubed":
        return clustered_box(134_217_728, 150_000, seed=5, nmax=2_000_000, star_fraction=0.15)
    raise KeyError(name)


def small_box(npart: int, nhalo: int, seed: int, nmax: int = 2000, **kw) -> ParticleSet:
    return clustered_box(npart, nhalo, seed=seed, nmax=nmax, **kw)


def halo_catalogue(nhalo: int, seed: int, nmin: int = 20, nmax: int = 2_000_000, slope: float = -1.9,
                   box: float = 100.0, total: int | None = None):
    """Already-grouped halos for the batched property stage.

    Returns (offsets int64[nhalo+1], pos (n,3), vel (n,3), mass (n,), density (n,))
    with members of halo h at [offsets[h], offsets[h+1]).  Positions are in
    box units of ``box`` (periodic, in [-box/2, box/2)); each halo's member
    density is an NFW-like decreasing function of radius so the densest
    member is near the centre.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    counts = _powerlaw_counts(rng, nhalo, slope, nmin, nmax)
    if total is not None:
        counts = np.maximum(nmin, np.floor(counts * (total / counts.sum()))).astype(np.int64)
    offsets = np.zeros(nhalo + 1, np.int64)
    np.cumsum(counts, out=offsets[1:])
    n = int(offsets[-1])
    pos = np.empty((n, 3), np.float64)
    vel = np.empty((n, 3), np.float64)
    dens = np.empty(n, np.float64)
    mass = np.full(n, 1.0, np.float64)
    for h in range(nhalo):
        a, b = int(offsets[h]), int(offsets[h + 1])
        k = b - a
        centre = (rng.random(3) - 0.5) * box
        rvir = 0.01 * box * (k / 1000.0) ** (1.0 / 3.0)
        r = _nfw_radius(rng, k, rvir)
        p = centre[None, :] + r[:, None] * _isotropic(rng, k)
        pos[a:b] = np.mod(p + 0.5 * box, box) - 0.5 * box
        sig = 100.0 * (k / 1000.0) ** (1.0 / 3.0)
        vel[a:b] = rng.normal(scale=sig, size=(k, 3)) + rng.normal(scale=300.0, size=3)[None, :]
        x = np.maximum(r / rvir, 1e-4)
        dens[a:b] = 1.0 / (x * (1 + 10 * x) ** 2) * (1.0 + 1e-3 * rng.random(k))
    return offsets, pos, vel, mass, dens
