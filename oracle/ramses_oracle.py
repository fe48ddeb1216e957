"""CPU restatement of the reference's RAMSES particle reader (test
infrastructure only: the checker of the GPU decoder, never the product).

Follows _read_ramses_new_1010 (src/input_output.py:624-760) and the counting /
loading passes of read_ramses_new_101 (src/input_output.py:856-989) with the
stellar payload off:
  * records per file: ncpu, ndim, npart, (localseed), nstar, (mstar_tot,
    mstar_lost), nsink, ndim position records, ndim velocity records, mass,
    id (int32), (level), Ra4: family (int8), (tag); then, when nstar > 0 or
    nsink > 0, Ra3 files hold the birth time (read to classify families);
  * families: Ra4 dm = family 1, star = family 2; Ra3 dm = id > 0 and birth
    time 0, star = (birth < 0 and id > 0) or (birth != 0 and id < 0)
    (input_output.py:697-703);
  * dense layout: ind = |id| (+ ndm for stars when family = all) - 1; a file
    whose selected ind leave [0, nselected) or repeat raises
    (input_output.py:712-728);
  * pos = x - 0.5, vel = v * scale_l / scale_t * 1e-5, mass = m
    (input_output.py:730-737); source_pid = |id| for a single family.
Pinned against the reference's own outputs (tests/golden/ramses_*.npz,
tests/golden/make_ramses_golden.py).
"""
from __future__ import annotations

import numpy as np


class Records:
    """Fortran sequential records (4-byte length before and after each)."""

    def __init__(self, path):
        self.buf = np.fromfile(path, np.uint8)
        self.off = 0

    def _next(self):
        n = int(self.buf[self.off:self.off + 4].view(np.uint32)[0])
        a = self.off + 4
        tail = int(self.buf[a + n:a + n + 4].view(np.uint32)[0])
        if tail != n:
            raise IOError(f"record sizes disagree: {n} vs {tail}")
        self.off = a + n + 4
        return a, n

    def read(self, dtype):
        a, n = self._next()
        return self.buf[a:a + n].view(dtype).copy()

    def skip(self, k=1):
        for _ in range(k):
            self._next()


def _file(path, version):
    R = Records(path)
    R.read(np.int32)  # ncpu
    ndim = int(R.read(np.int32)[0])
    npart = int(R.read(np.int32)[0])
    R.skip(1)
    nstar = int(R.read(np.int32)[0])
    R.skip(2)
    nsink = int(R.read(np.int32)[0])
    pos = np.stack([R.read(np.float64) for _ in range(ndim)], 1)
    vel = np.stack([R.read(np.float64) for _ in range(ndim)], 1)
    mass = R.read(np.float64)
    idp = R.read(np.int32)
    R.skip(1)
    fam = None
    if version == 4:
        fam = R.read(np.int8)
        R.skip(1)
    tmpt = None
    if (nstar > 0 or nsink > 0) and version != 4:
        tmpt = R.read(np.float64)
    if version == 4:
        dm, star = fam == 1, fam == 2
    else:
        if tmpt is None:
            tmpt = np.zeros(npart)
        dm = (idp > 0) & (tmpt == 0)
        star = ((tmpt < 0) & (idp > 0)) | ((tmpt != 0) & (idp < 0))
    return pos, vel, mass, idp, dm, star


def read_parts(paths, version, family="all", scale_l=1.0, scale_t=1.0):
    files = [_file(p, version) for p in paths]
    ndm = sum(int(np.count_nonzero(f[4])) for f in files)
    nstar = sum(int(np.count_nonzero(f[5])) for f in files)
    sel = {"all": ndm + nstar, "dm": ndm, "star": nstar}[family]
    off_star = ndm if family == "all" else 0
    pos = np.empty((sel, 3))
    vel = np.empty((sel, 3))
    mass = np.empty(sel)
    spid = np.full(sel, -1, np.int64)
    for k, (p, v, m, idp, dm, star) in enumerate(files):
        mask = dm | star if family == "all" else (dm if family == "dm" else star)
        src = np.abs(idp).astype(np.int64)
        loc = np.where(star, src + off_star, src) if family == "all" else src
        ind = loc[mask] - 1
        if np.any(ind < 0) or np.any(ind >= sel) or len(np.unique(ind)) != len(ind):
            raise RuntimeError(f"non-dense or duplicate {family} particle ids in file {k + 1}")
        pos[ind] = p[mask] - 0.5
        vel[ind] = v[mask] * scale_l / scale_t * 1e-5
        mass[ind] = m[mask]
        spid[ind] = src[mask]
    out = dict(pos=pos, vel=vel, mass=mass, ndm=ndm, nstar=nstar, nselected=sel)
    if family != "all":
        out["source_pid"] = spid
    return out
