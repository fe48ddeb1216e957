"""The device RAMSES decoder (ahop_ramses_*) against the reference's own
reader outputs (tests/golden/ramses_*.npz), bit for bit, and its errors on
files the reference rejects: an id repeated inside a file, an id outside the
dense layout, a record whose two lengths disagree, a missing file."""
import glob
import os
import sys

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = sorted(glob.glob(os.path.join(HERE, "golden", "ramses_*_*.npz")))
sys.path.insert(0, os.path.join(HERE, "golden"))
import ramses_files  # noqa: E402
import ramses_oracle  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from ahop_b200 import build
    build.build()


def _files(tmp_path, g):
    return ramses_files.write_case(str(tmp_path), int(g["w_seed"]), int(g["w_version"]), int(g["w_ncpu"]),
                                   int(g["w_ndm"]), int(g["w_nstar"]), int(g["w_nother"]))


@pytest.mark.parametrize("path", GOLD, ids=[os.path.basename(p)[:-4] for p in GOLD])
def test_decoder_matches_reference(tmp_path, path):
    from ahop_b200 import ramses
    g = np.load(path)
    paths = _files(tmp_path, g)
    fam = str(g["family"])
    r = ramses.read_parts(os.path.dirname(paths[0]), int(g["w_version"]), fam, float(g["scale_l"]),
                          float(g["scale_t"]))
    assert (r["ndm"], r["nstar"], r["nselected"]) == (int(g["ndm"]), int(g["nstar"]), int(g["nselected"]))
    for k in ("pos", "vel", "mass"):
        assert np.array_equal(r[k].cpu().numpy(), g[k]), k
    if fam != "all":
        assert np.array_equal(r["source_pid"].cpu().numpy(), g["source_pid"])


def _id_record(path):
    R = ramses_oracle.Records(path)
    R.skip(8 + 7)
    a, n = R._next()
    return R, R.buf[a:a + n].view(np.int32)


def test_decoder_rejects_what_the_reference_rejects(tmp_path):
    from ahop_b200 import AhopError, ramses
    g = np.load(os.path.join(HERE, "golden", "ramses_ra3_dmonly_all.npz"))  # every particle is dark matter
    v = int(g["w_version"])
    # an id repeated inside one file
    paths = _files(tmp_path / "a", g)
    R, ids = _id_record(paths[1])
    ids[1] = ids[0]
    R.buf.tofile(paths[1])
    with pytest.raises(RuntimeError):
        ramses_oracle.read_parts(paths, v, "all")
    with pytest.raises(AhopError, match="EDATA.*icpu=2"):
        ramses.read_parts(paths, v, "all")
    # an id past the dense layout
    paths = _files(tmp_path / "b", g)
    R, ids = _id_record(paths[0])
    ids[0] = 10 ** 8
    R.buf.tofile(paths[0])
    with pytest.raises(RuntimeError):
        ramses_oracle.read_parts(paths, v, "all")
    with pytest.raises(AhopError, match="EDATA.*icpu=1"):
        ramses.read_parts(paths, v, "all")
    # a record whose trailing length disagrees with its leading one
    paths = _files(tmp_path / "c", g)
    R, ids = _id_record(paths[0])
    a = R.off - 4
    R.buf[a:a + 4] = np.array([7], np.uint32).view(np.uint8)
    R.buf.tofile(paths[0])
    with pytest.raises(AhopError, match="EDATA.*Sizes do not agree"):
        ramses.read_parts(paths, v, "all")
    # a missing file
    with pytest.raises(AhopError, match="EIO"):
        ramses.read_parts([str(tmp_path / "none" / "part_00001.out00001")], v, "all")


def test_snapshot_from_files_matches_host_arrays(tmp_path):
    """run_snapshot_files (device decode straight into the pipeline) equals
    run_snapshot on the same particles taken from the reference fixture."""
    from ahop_b200 import halo_props, pipeline
    g = np.load(os.path.join(HERE, "golden", "ramses_ra4_all.npz"))
    paths = _files(tmp_path, g)
    halo_props.set_tiles([256] * halo_props.BUCKETS)
    try:
        a = pipeline.run_snapshot_files(os.path.dirname(paths[0]), 4, "all", float(g["scale_l"]),
                                        float(g["scale_t"]), epot=3)
        b = pipeline.run_snapshot(g["pos"], g["vel"], g["mass"], epot=3)
    finally:
        halo_props.set_tiles(None)
    assert a["nselected"] == int(g["nselected"])
    assert np.array_equal(a["ids"], b["ids"]) and np.array_equal(a["offsets"], b["offsets"])
    assert np.array_equal(a["props"], b["props"], equal_nan=True)


def test_decoder_reads_an_empty_file(tmp_path):
    """A cpu file without particles: no payload copies, no scatter launch; the
    rows equal the restatement's."""
    from ahop_b200 import ramses
    P = ramses_files.make_particles(44, 4, 500, 120, 30)
    n = len(P["mass"])
    paths = ramses_files.write_arrays(str(tmp_path), P, 4, [0, 0, n // 2, n])
    for fam in ("all", "dm", "star"):
        r = ramses.read_parts(paths, 4, fam, 2.0, 3.0)
        o = ramses_oracle.read_parts(paths, 4, fam, 2.0, 3.0)
        assert r["nselected"] == o["nselected"]
        for k in ("pos", "vel", "mass"):
            assert np.array_equal(r[k].cpu().numpy(), o[k]), (fam, k)
