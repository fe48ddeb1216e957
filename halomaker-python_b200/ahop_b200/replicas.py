"""Several GPUs: one process per GPU, torch.distributed for the plumbing.

The finder does not shard (its structure tree needs a global merge over the
whole box), so snapshots run as independent replicas, one per rank, timed as
the maximum over ranks.  The batched halo properties do shard: halos are
independent, so each rank takes a contiguous run of halos of about equal cost
(the direct potential makes a halo of n members cost ~n^2), computes its rows
on its own GPU, and rank 0 gathers the rows in halo order -- the one exchange.
The same code runs on the gloo backend for tests on CPU.
"""
from __future__ import annotations

import numpy as np


def halo_cost(off) -> np.ndarray:
    """Work of each halo: the O(n) reductions plus the n(n-1)/2 pair sum."""
    n = np.diff(np.asarray(off, np.int64)).astype(np.float64)
    return n + 0.5 * n * (n - 1.0)


def partition_halos(off, nparts: int) -> np.ndarray:
    """Split halos into nparts contiguous runs of about equal cost.

    Returns bounds b (nparts + 1 halo indices): part p owns halos [b[p], b[p+1]).
    Cuts are placed at the halo where the cumulative cost crosses p/nparts of
    the total, so a single very large halo is never split (it cannot be).
    """
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    nh = len(off) - 1
    c = np.cumsum(halo_cost(off))
    total = c[-1] if nh else 0.0
    b = np.zeros(nparts + 1, np.int64)
    b[-1] = nh
    for p in range(1, nparts):
        b[p] = int(np.searchsorted(c, total * p / nparts, side="left")) if nh else 0
        b[p] = min(max(b[p], b[p - 1]), nh)
    return b


def local_members(off, bounds, rank):
    """Member offsets (rebased) and the member range of this rank's halos."""
    off = np.asarray(off, np.int64)
    h0, h1 = int(bounds[rank]), int(bounds[rank + 1])
    m0, m1 = int(off[h0]), int(off[h1])
    return off[h0:h1 + 1] - m0, m0, m1


def max_over_ranks(x: float, dist=None) -> float:
    """The largest value over all ranks (timings are taken as the slowest rank)."""
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_rows(rows: np.ndarray, bounds, dist, root: int = 0):
    """Gather each rank's (nlocal, nfields) rows to `root` in halo order.

    Every rank passes its own block (ranks own contiguous halo runs given by
    bounds); blocks are padded to the longest so one all_gather carries them.
    Returns the (nhalo, nfields) array on root and None elsewhere.
    """
    import torch
    world = dist.get_world_size()
    rank = dist.get_rank()
    counts = np.diff(np.asarray(bounds, np.int64))
    nf = rows.shape[1]
    width = int(counts.max()) if len(counts) else 0
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    buf = torch.zeros((max(width, 1), nf), dtype=torch.float64, device=dev)
    if len(rows):
        buf[:len(rows)] = torch.from_numpy(np.ascontiguousarray(rows, np.float64)).to(dev)
    parts = [torch.zeros_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    if rank != root:
        return None
    return np.concatenate([parts[r][:counts[r]].cpu().numpy() for r in range(world)], 0)
