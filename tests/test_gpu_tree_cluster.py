"""Structure tree with wide tasks on thread-block clusters vs one CTA per task.

A wide task's cluster splits the union, root-finding and group-term passes of
every level over its CTAs (the leader's union-find array in distributed
shared memory).  The grouping it computes does not depend on how the positions
are split, so the finder's outputs must be the same bit for bit with
clusters of 4 CTAs and with one CTA per task; the parity tests compare the
default (clusters) with the oracle.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from ahop_b200 import build
    build.build()


def _run(lib, finder, ps, ctas):
    from ahop_b200 import _lib as L
    lib.ahop_debug_set_tree_cluster.argtypes = [C.c_int32]
    L.check(lib.ahop_debug_set_tree_cluster(ctas), "set_tree_cluster")
    out = finder.run(ps.pos, ps.mass)
    return out, lib.ahop_debug_get_tree_cluster()


def test_cluster_and_single_cta_trees_are_identical():
    from ahop_b200 import _lib as L, finder, synthetic
    lib = L.lib()
    # halos large enough for tasks of more than 512 groups (the wide path)
    ps = synthetic.clustered_box(1_048_576, 1_200, seed=11, nmax=150_000)
    finder.configure(ps.n)
    try:
        one, k1 = _run(lib, finder, ps, 1)
        four, k4 = _run(lib, finder, ps, 4)
        again, _ = _run(lib, finder, ps, 4)
    finally:
        lib.ahop_debug_set_tree_cluster(4)
    assert k1 == 1
    assert k4 == 4, "a B200 holds a cluster of 4 wide CTAs"
    assert one["nnodes"] > 100
    for key in ("density", "liste_parts", "integer_table", "real_table"):
        assert np.array_equal(one[key], four[key]), key
        assert np.array_equal(four[key], again[key]), key


def test_wide_tasks_with_global_union_find_are_identical():
    """Wide tasks larger than the shared union-find array keep their parents in
    global memory (followers then union there too); capping the array forces
    that path on a small box."""
    from ahop_b200 import _lib as L, finder, synthetic
    lib = L.lib()
    lib.ahop_debug_set_tree_par_cap.argtypes = [C.c_int32]
    ps = synthetic.clustered_box(1_048_576, 1_200, seed=11, nmax=150_000)
    finder.configure(ps.n)
    ref = finder.run(ps.pos, ps.mass)
    try:
        L.check(lib.ahop_debug_set_tree_par_cap(600), "set_tree_par_cap")
        four, _ = _run(lib, finder, ps, 4)
        one, _ = _run(lib, finder, ps, 1)
    finally:
        lib.ahop_debug_set_tree_par_cap(0)
        lib.ahop_debug_set_tree_cluster(4)
    for key in ("density", "liste_parts", "integer_table", "real_table"):
        assert np.array_equal(ref[key], four[key]), key
        assert np.array_equal(ref[key], one[key]), key
