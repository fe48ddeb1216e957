"""The tree-brick catalogue writer against the reference's own writer.

tests/golden/treebrick_case.npz (tests/golden/make_treebrick_golden.py)
records write_tree_brick_hdf (src/input_output.py:1048-1269) through a
recording stand-in for h5py, on catalogue records made by the reference's
init_halos_16 from an MSM tree.  Here the same inputs go through
ahop_b200.tree_bricks: the halo/subhalo tree fields must equal
init_halos_16's records byte for byte, and the writer must make the same
calls in the same order with the same attribute types and values and
byte-identical datasets (unit conversion included).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
import h5py_record  # noqa: E402

GOLD = os.path.join(HERE, "golden", "treebrick_case.npz")


def _meta(d):
    out = {}
    for k, (t, v) in json.loads(str(d["meta"])).items():
        out[k] = {"float64": np.float64, "float": float, "int": int, "bool": bool, "str": str}[t](v)
    return out


def test_tree_fields_match_init_halos_16():
    from ahop_b200 import tree_bricks as T
    d = np.load(GOLD)
    assert T.HALO_DTYPE == d["tree"].dtype
    cat = T.new_catalogue(len(d["level"]))
    T.init_tree_fields(cat, d["level"], d["mother"], d["first_sister"], d["first_daughter"], numstep=7)
    assert cat.tobytes() == d["tree"].tobytes()
    assert (cat["level"] > 1).any() and (cat["nbsub"] > 0).any()


def test_writer_matches_the_reference_writer(tmp_path):
    from ahop_b200 import tree_bricks as T
    d = np.load(GOLD)
    f = h5py_record.File(str(tmp_path / "tb.h5"), "w")
    T.write(f, _meta(d), d["records"], d["member_index"], d["member_count"], d["pids0_groupsorted"])
    log, arrays = h5py_record.record_of(f)
    ref = json.loads(str(d["log"]))
    assert [(e["op"], e["path"], e.get("name")) for e in log] == [(e["op"], e["path"], e.get("name")) for e in ref]
    for a, b in zip(log, ref):
        assert {k: v for k, v in a.items() if k != "data"} == {k: v for k, v in b.items() if k != "data"}, a["path"]
        if a.get("data") is not None:
            x, y = arrays[a["data"]], d["rec_" + b["data"]]
            assert x.dtype == y.dtype and x.shape == y.shape and x.tobytes() == y.tobytes(), a["path"]
