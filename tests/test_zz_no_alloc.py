"""The allocation-free halo-property entry point (ahop_halo_props_noalloc).

Some callers cannot allocate device memory while they run -- e.g. code that
executes while another part of the process captures a CUDA graph, or a host
framework that owns all device memory through its own pool.  For them the
library offers one entry point whose scratch lives in a fixed-size device
array compiled into the library.  This test calls it through the C ABI twice
in a row and checks it against the allocating entry point
(ahop_halo_props_device) with the tolerances of the other halo-property tests
(the two entry points sum members and FP32 pairs in other groups), and checks
that sizes beyond its stated limits are rejected.  It sits in its
own file that pytest collects last and passes alone or after the other tests.
"""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

FIELDS_RTOL = 1e-12
FP32C_RTOL = 1e-6
FP32C_FIELDS = ("ep32c", "spin32c")
# sums with cancellation (angular momentum, off-diagonal inertia) and what
# derives from them: the two entry points sum members in other groups (the
# allocating one cuts large halos into chunks), so these get the tolerances
# the other halo-property tests use against the oracle
CANCEL_FIELDS = ("Lx", "Ly", "Lz", "Ixy", "Ixz", "Iyz")
DERIVED_RTOL = {"sha": 1e-9, "shb": 1e-9, "shc": 1e-9, "spin64": 1e-10}


@pytest.fixture(scope="module")
def catalogue():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from ahop_b200 import build, synthetic
    build.build()
    return synthetic.halo_catalogue(300, seed=91, nmin=20, nmax=30000, box=100.0)


def test_noalloc_matches_allocating_entry_point_twice(catalogue):
    import torch
    from ahop_b200 import halo_props
    off, pos, vel, mass, dens = catalogue
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    d_off, d_pos, d_vel, d_mass, d_dens = t(off), t(pos), t(vel), t(mass), t(dens)
    nh = len(off) - 1
    ref = torch.zeros((nh, halo_props.NF), dtype=torch.float64, device=dev)
    halo_props.compute_device(d_off, d_pos, d_vel, d_mass, d_dens, ref, 100.0, 70.0)
    torch.cuda.synchronize()
    r = ref.cpu().numpy()
    for call in range(2):
        out = torch.full((nh, halo_props.NF), np.nan, dtype=torch.float64, device=dev)
        halo_props.compute_device_noalloc(d_off, d_pos, d_vel, d_mass, d_dens, out, 100.0, 70.0)
        torch.cuda.synchronize()
        o = out.cpu().numpy()
        for k, name in enumerate(halo_props.FIELDS):
            rtol = FP32C_RTOL if name in FP32C_FIELDS else DERIVED_RTOL.get(name, FIELDS_RTOL)
            atol = 0.0
            if name in CANCEL_FIELDS:
                rtol, atol = 1e-10, 1e-12 * np.abs(r[:, k]).max()
            np.testing.assert_allclose(o[:, k], r[:, k], rtol=rtol, atol=atol, err_msg=f"call {call}: {name}")


def test_noalloc_rejects_sizes_beyond_its_limit(catalogue):
    import torch
    from ahop_b200 import AhopError, halo_props
    dev = torch.device("cuda:0")
    nh = 65537  # one more halo than the fixed scratch holds
    d_off = torch.arange(nh + 1, dtype=torch.int64, device=dev)
    z3 = torch.zeros((nh, 3), dtype=torch.float64, device=dev)
    z1 = torch.ones(nh, dtype=torch.float64, device=dev)
    out = torch.zeros((nh, halo_props.NF), dtype=torch.float64, device=dev)
    with pytest.raises(AhopError, match="exceeds the maximum"):
        halo_props.compute_device_noalloc(d_off, z3, z3, z1, z1, out, 100.0, 70.0)
