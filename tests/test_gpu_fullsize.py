"""The full 256^3 workload (16,777,216 particles, 19,200 halos, seed 2): the
CUDA finder's module outputs against the CPU oracle, bit for bit.

This is the size the throughput is quoted on, so every branch the smaller
parity cases may miss at scale (deep structure-tree chains, colours with
thousands of groups, groups with millions of members, undecided significance
tests) is exercised here.  The oracle runs on all host cores (~30 s).
"""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

import oracle  # noqa: E402


@pytest.fixture(scope="module", autouse=True)
def _built():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from ahop_b200 import build
    build.build()


def test_256cubed_matches_oracle():
    from ahop_b200 import finder, synthetic
    ps = synthetic.workload("c2_256cubed")
    finder.configure(ps.n)
    out = finder.run(ps.pos, ps.mass)
    ref = oracle.run(ps.pos, ps.mass, oracle.default_params(ps.n))
    assert np.array_equal(out["density"], ref["density"])
    assert out["nnodes"] == ref["nnodes"] > 10000
    assert np.array_equal(out["integer_table"], ref["integer_table"])
    assert np.array_equal(out["real_table"], ref["real_table"])
    assert np.array_equal(out["liste_parts"], ref["liste_parts"])
