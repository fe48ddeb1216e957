"""The allocation-free halo-property entry point (ahop_halo_props_noalloc).

Some callers cannot allocate device memory while they run -- e.g. code that
executes while another part of the process captures a CUDA graph, or a host
framework that owns all device memory through its own pool.  For them the
library offers one entry point whose scratch lives in a fixed-size device
array compiled into the library.  This test calls it through the C ABI twice
in a row and checks it against the allocating entry point
(ahop_halo_props_device) with the tolerances of the other halo-property tests
(the two entry points sum members and FP32 pairs in other groups), and checks
that sizes beyond its stated limits are rejected (the halo count on the
host, the work-item count on the device), that a capturing stream is refused,
and that a call allocates no device memory.  It sits in its own file that
pytest collects last and passes alone or after the other tests.
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


@pytest.fixture(scope="module")
def device_case(catalogue):
    """The catalogue on the device and the allocating entry point's rows."""
    import torch
    from ahop_b200 import halo_props
    off, pos, vel, mass, dens = catalogue
    dev = torch.device("cuda:0")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    args = (t(off), t(pos), t(vel), t(mass), t(dens))
    nh = len(off) - 1
    ref = torch.zeros((nh, halo_props.NF), dtype=torch.float64, device=dev)
    halo_props.compute_device(*args, ref, 100.0, 70.0)
    torch.cuda.synchronize()
    return args, nh, ref.cpu().numpy()


def _check_noalloc(device_case, label):
    import torch
    from ahop_b200 import halo_props
    args, nh, r = device_case
    out = torch.full((nh, halo_props.NF), np.nan, dtype=torch.float64, device=args[0].device)
    halo_props.compute_device_noalloc(*args, out, 100.0, 70.0)
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    for k, name in enumerate(halo_props.FIELDS):
        rtol = FP32C_RTOL if name in FP32C_FIELDS else DERIVED_RTOL.get(name, FIELDS_RTOL)
        atol = 0.0
        if name in CANCEL_FIELDS:
            rtol, atol = 1e-10, 1e-12 * np.abs(r[:, k]).max()
        np.testing.assert_allclose(o[:, k], r[:, k], rtol=rtol, atol=atol, err_msg=f"{label}: {name}")


def test_noalloc_matches_allocating_entry_point_twice(device_case):
    for call in range(2):
        _check_noalloc(device_case, f"call {call}")


def test_noalloc_allocates_no_device_memory(device_case):
    import torch
    from ahop_b200 import halo_props
    args, nh, _ = device_case
    _check_noalloc(device_case, "warm-up call")
    # the rows buffer comes from torch's pool before the call is measured
    out = torch.zeros((nh, halo_props.NF), dtype=torch.float64, device=args[0].device)
    torch.cuda.synchronize()
    free1, alloc1 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
    halo_props.compute_device_noalloc(*args, out, 100.0, 70.0)
    torch.cuda.synchronize()
    free2, alloc2 = torch.cuda.mem_get_info()[0], torch.cuda.memory_allocated()
    assert alloc2 == alloc1, "torch's allocator saw an allocation during the call"
    assert free2 == free1, f"device free memory changed by {free1 - free2} bytes during the call"


def test_noalloc_rejects_sizes_beyond_its_limit(device_case):
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


def test_noalloc_rejects_work_items_beyond_its_limit(device_case):
    """One halo of 262,145 x 256 members needs one work item more than the
    array holds; the device-side count rejects the call before any member is
    read (the member arrays here are a few elements long), and the next
    valid call still matches."""
    import torch
    from ahop_b200 import AhopError, halo_props
    dev = torch.device("cuda:0")
    d_off = torch.tensor([0, 262145 * 256], dtype=torch.int64, device=dev)
    z3 = torch.zeros((4, 3), dtype=torch.float64, device=dev)
    z1 = torch.ones(4, dtype=torch.float64, device=dev)
    out = torch.zeros((1, halo_props.NF), dtype=torch.float64, device=dev)
    with pytest.raises(AhopError, match="work items"):
        halo_props.compute_device_noalloc(d_off, z3, z3, z1, z1, out, 100.0, 70.0)
    _check_noalloc(device_case, "after the rejected call")


def test_noalloc_refuses_a_capturing_stream(device_case):
    import torch
    from ahop_b200 import AhopError, halo_props
    args, nh, _ = device_case
    out = torch.zeros((nh, halo_props.NF), dtype=torch.float64, device=args[0].device)
    x = torch.zeros(8, device=args[0].device)
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    with torch.cuda.graph(g, stream=s):
        x.add_(1.0)
        with pytest.raises(AhopError, match="captured"):
            halo_props.compute_device_noalloc(*args, out, 100.0, 70.0, stream=s)
    g.replay()
    torch.cuda.synchronize()
    assert float(x.sum()) == 8.0
    del g
    _check_noalloc(device_case, "after the refused capture")
