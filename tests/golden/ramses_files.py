"""Synthetic RAMSES particle files for the reader tests.

No simulation output is available, so the tests write their own part files
in the layout the reference's reader expects (_read_ramses_new_1010,
src/input_output.py:624-760): Fortran sequential records framed by 4-byte
lengths, per file

    ncpu, ndim, npart, localseed, nstar_tot, mstar_tot, mstar_lost, nsink,
    x, y, z, vx, vy, vz, mass, id (int32), level (int32),
    [Ra4] family (int8), tag (int8),
    [if nstar_tot > 0 or nsink > 0] birth time (float64), metallicity (float64).

Families: in Ra4 files the family record says it (1 = dark matter, 2 = star,
other codes are neither); in Ra3 files dark matter has id > 0 and birth time
0, a star has a negative birth time (id > 0) or a non-zero one with id < 0,
and id < 0 with birth time 0 is neither.  Dark-matter ids and star ids are
each dense (1..ndm, 1..nstar), the particles shuffled over the files.
"""
from __future__ import annotations

import os

import numpy as np


def _rec(f, arr):
    a = np.ascontiguousarray(arr)
    n = np.array([a.nbytes], np.uint32)
    f.write(n.tobytes())
    f.write(a.tobytes())
    f.write(n.tobytes())


def make_particles(seed: int, version: int, ndm: int, nstar: int, nother: int):
    """Particle table (all files together, shuffled): dict of arrays."""
    rng = np.random.Generator(np.random.PCG64(seed))
    n = ndm + nstar + nother
    kind = np.concatenate([np.ones(ndm, np.int8), np.full(nstar, 2, np.int8), np.full(nother, 3, np.int8)])
    ids = np.concatenate([np.arange(1, ndm + 1), np.arange(1, nstar + 1),
                          np.arange(1, nother + 1)]).astype(np.int32)
    tbirth = np.zeros(n)
    if version == 3:
        # stars: half with id > 0 and a negative birth time, half with id < 0 and a non-zero one
        st = np.flatnonzero(kind == 2)
        neg = st[: len(st) // 2]
        pos_ = st[len(st) // 2:]
        tbirth[neg] = -rng.uniform(0.1, 5.0, len(neg))
        ids[pos_] = -ids[pos_]
        tbirth[pos_] = rng.uniform(-5.0, 5.0, len(pos_))
        tbirth[pos_[tbirth[pos_] == 0]] = 1.0
        # neither: id < 0 and birth time 0
        ids[kind == 3] = -ids[kind == 3]
    fam = np.where(kind == 1, 1, np.where(kind == 2, 2, rng.choice(np.array([0, 3, 4, -2], np.int8), n)))
    fam = fam.astype(np.int8)
    perm = rng.permutation(n)
    pos = rng.random((n, 3))
    vel = rng.normal(scale=0.05, size=(n, 3))
    mass = np.where(kind == 2, 1e-7, 1e-6) * rng.uniform(0.9, 1.1, n)
    level = rng.integers(5, 12, n).astype(np.int32)
    metal = rng.uniform(0.0, 0.02, n)
    return dict(pos=pos[perm], vel=vel[perm], mass=mass[perm], id=ids[perm], fam=fam[perm], tbirth=tbirth[perm],
                level=level[perm], metal=metal[perm], kind=kind[perm])


def write_case(root: str, seed: int, version: int, ncpu: int, ndm: int, nstar: int, nother: int,
               nchar: str = "00001") -> list:
    """Write part_<nchar>.out000NN (NN = 1..ncpu) under root/output_<nchar>/;
    returns the file paths in cpu order."""
    P = make_particles(seed, version, ndm, nstar, nother)
    n = len(P["mass"])
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    cuts = np.sort(rng.integers(0, n + 1, ncpu - 1))
    bounds = np.concatenate([[0], cuts, [n]])
    return write_arrays(root, P, version, bounds, seed, nchar)


def write_arrays(root: str, P: dict, version: int, bounds, seed: int = 0, nchar: str = "00001") -> list:
    """Write the particle table P (make_particles' keys) as part files, file c
    holding rows [bounds[c], bounds[c+1])."""
    ncpu = len(bounds) - 1
    out = os.path.join(root, f"output_{nchar}")
    os.makedirs(out, exist_ok=True)
    paths = []
    nstar_tot = int(np.count_nonzero(P["kind"] == 2))
    for c in range(ncpu):
        a, b = int(bounds[c]), int(bounds[c + 1])
        path = os.path.join(out, f"part_{nchar}.out{c + 1:05d}")
        with open(path, "wb") as f:
            _rec(f, np.array([ncpu], np.int32))
            _rec(f, np.array([3], np.int32))
            _rec(f, np.array([b - a], np.int32))
            _rec(f, np.arange(4, dtype=np.int32) + seed)          # localseed
            _rec(f, np.array([nstar_tot], np.int32))
            _rec(f, np.array([1.5e-3]))                           # mstar_tot
            _rec(f, np.array([0.0]))                              # mstar_lost
            _rec(f, np.array([0], np.int32))                      # nsink
            for d in range(3):
                _rec(f, P["pos"][a:b, d])
            for d in range(3):
                _rec(f, P["vel"][a:b, d])
            _rec(f, P["mass"][a:b])
            _rec(f, P["id"][a:b])
            _rec(f, P["level"][a:b])
            if version == 4:
                _rec(f, P["fam"][a:b])
                _rec(f, np.zeros(b - a, np.int8))                 # tag
            if nstar_tot > 0:
                _rec(f, P["tbirth"][a:b])
                _rec(f, P["metal"][a:b])
        paths.append(path)
    return paths


# the cases the golden fixtures and the tests share
CASES = [
    dict(name="ra3", seed=41, version=3, ncpu=4, ndm=3000, nstar=700, nother=150),
    dict(name="ra4", seed=42, version=4, ncpu=3, ndm=2500, nstar=900, nother=200),
    dict(name="ra3_dmonly", seed=43, version=3, ncpu=2, ndm=1800, nstar=0, nother=0),
]
SCALE_L, SCALE_T = 3.0e24, 4.5e17
