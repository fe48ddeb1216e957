"""The reference driver's own calls on the f2py module, replayed on CPU.

tests/golden/dropin_calls.npz holds what src/compute_neiKDtree_mod.py passes
to ``neikdtree`` when it runs with H.FORTRAN = True (init_adaptahop_130 ->
compute_adaptahop_131, recorded by tests/golden/make_dropin_golden.py).  This
checks that the Python mirror of the module offers every subroutine the
driver calls with the arity it uses, and replays the three parameter calls
(host-only: they store parameters) with the recorded argument types.  The
compute call itself is replayed on the GPU (test_gpu_dropin.py).
"""
import inspect
import json
import os

import numpy as np
import pytest

REC = os.path.join(os.path.dirname(__file__), "golden", "dropin_calls.npz")


def load_calls():
    d = np.load(REC)
    calls = json.loads(str(d["calls"]))
    out = []
    for c in calls:
        args = []
        for a in c["args"]:
            if a["type"] == "ndarray":
                arr = d[a["key"]]
                arr = np.asfortranarray(arr) if a["f_contiguous"] and not a["c_contiguous"] else arr
                args.append(arr)
            elif a["type"] in ("float64", "float32"):
                args.append(getattr(np, a["type"])(a["value"]))
            elif a["type"] in ("int32", "int64"):
                args.append(getattr(np, a["type"])(a["value"]))
            elif a["type"] == "bool_":
                args.append(np.bool_(a["value"]))
            else:
                args.append({"int": int, "float": float, "bool": bool, "str": str}[a["type"]](a["value"]))
        out.append((c["name"], args, c["args"]))
    return out


def test_recorded_sequence_is_the_reference_drivers():
    calls = load_calls()
    assert [c[0] for c in calls] == ["sync_from_init_adaptahop", "sync_from_change_pos", "sync_others",
                                     "compute_adaptahop", "close"]
    pos, mass = calls[3][1]
    meta = calls[3][2]
    assert meta[0]["f_contiguous"] and pos.shape[0] == 3 and pos.dtype == np.float64
    assert mass.shape == (pos.shape[1],)
    # change_pos_1310 scaled the positions by boxsize2 (NEI:205)
    box = calls[1][1][4]
    assert box == 100.0 and np.abs(pos).max() <= box / 2 and np.abs(pos).max() > box / 4


def test_mirror_accepts_every_recorded_call():
    from compute_adaptahop import neikdtree
    for name, args, _ in load_calls():
        fn = getattr(neikdtree, name)
        params = inspect.signature(fn).parameters
        assert len(params) == len(args), name


def test_parameter_calls_replay_on_the_host():
    from compute_adaptahop import neikdtree
    for name, args, _ in load_calls()[:3]:
        getattr(neikdtree, name)(*args)
    # a wrong argument count fails in the mirror like an f2py call would
    name, args, _ = load_calls()[1]
    with pytest.raises(TypeError):
        neikdtree.sync_from_change_pos(*args[:-1])
