"""The RAMSES reader restatement (oracle/ramses_oracle.py) against the
reference's own reader outputs (tests/golden/ramses_*.npz, made by
tests/golden/make_ramses_golden.py from the files tests/golden/ramses_files.py
writes), bit for bit, and its error behaviour on a repeated id."""
import glob
import os

import numpy as np
import pytest

import ramses_oracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = sorted(glob.glob(os.path.join(HERE, "golden", "ramses_*_*.npz")))


def _files(tmp_path, g):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import ramses_files
    return ramses_files.write_case(str(tmp_path), int(g["w_seed"]), int(g["w_version"]), int(g["w_ncpu"]),
                                   int(g["w_ndm"]), int(g["w_nstar"]), int(g["w_nother"]))


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_oracle_matches_reference(tmp_path, path):
    g = np.load(path)
    paths = _files(tmp_path, g)
    r = ramses_oracle.read_parts(paths, int(g["w_version"]), str(g["family"]), float(g["scale_l"]),
                                 float(g["scale_t"]))
    assert (r["ndm"], r["nstar"], r["nselected"]) == (int(g["ndm"]), int(g["nstar"]), int(g["nselected"]))
    for k in ("pos", "vel", "mass"):
        assert np.array_equal(r[k], g[k]), k
    if str(g["family"]) != "all":
        assert np.array_equal(r["source_pid"], g["source_pid"])


def test_oracle_rejects_repeated_id_in_a_file(tmp_path):
    g = np.load(os.path.join(HERE, "golden", "ramses_ra3_dmonly_all.npz"))  # every particle is dark matter
    paths = _files(tmp_path, g)
    ramses_oracle_repeat_id(paths[1])
    with pytest.raises(RuntimeError, match="duplicate"):
        ramses_oracle.read_parts(paths, int(g["w_version"]), "all", 1.0, 1.0)


def ramses_oracle_repeat_id(path):
    """Give the second selected particle of a file the first one's id (in place)."""
    R = ramses_oracle.Records(path)
    R.skip(3 + 5)
    for _ in range(7):
        R.skip()
    a, n = R._next()
    ids = R.buf[a:a + n].view(np.int32)
    pos = np.flatnonzero(ids > 0)[:2]
    ids[pos[1]] = ids[pos[0]]
    R.buf.tofile(path)


def test_oracle_reads_an_empty_file(tmp_path):
    """A cpu file without particles (npart = 0, empty records) contributes nothing."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import ramses_files
    P = ramses_files.make_particles(44, 4, 500, 120, 30)
    n = len(P["mass"])
    paths = ramses_files.write_arrays(str(tmp_path), P, 4, [0, 0, n // 2, n])
    r = ramses_oracle.read_parts(paths, 4, "all")
    full = ramses_oracle.read_parts(ramses_files.write_arrays(str(tmp_path / "one"), P, 4, [0, n]), 4, "all")
    assert r["nselected"] == 620
    for k in ("pos", "vel", "mass"):
        assert np.array_equal(r[k], full[k])
