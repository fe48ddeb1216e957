"""CPU restatement of the MSM halo/subhalo selection -- TEST INFRASTRUCTURE ONLY.

Follows select_with_MS_method_1319 (src/compute_neiKDtree_mod.py:260-464)
step by step on the finder's tables (real_table (nnodes, 8), integer_table
(nnodes, 6), node k+1 in row k) and membership, and the member grouping of
compute_adaptahop_131 (NEI:107-119).  Pinned against fixtures made by the
reference itself (tests/golden/make_msm_golden.py).
"""
from __future__ import annotations

import numpy as np


def select_msm(real_table, integer_table, liste_parts):
    nn = integer_table.shape[0]
    mass = np.zeros(nn + 1, np.int64)
    level = np.zeros(nn + 1, np.int64)
    mother = np.zeros(nn + 1, np.int64)
    firstchild = np.zeros(nn + 1, np.int64)
    sister = np.zeros(nn + 1, np.int64)
    truemass = np.zeros(nn + 1)
    mass[1:], level[1:], mother[1:] = integer_table[:, 0], integer_table[:, 1], integer_table[:, 2]
    firstchild[1:], sister[1:] = integer_table[:, 3], integer_table[:, 5]
    truemass[1:] = real_table[:, 4]
    # own mass: subtract the children (NEI:266-281), children read before they change
    m1, t1 = mass.copy(), truemass.copy()
    for i in range(1, nn + 1):
        c = firstchild[i]
        if c <= 0:
            continue
        while c > 0:
            m1[i] -= mass[c]
            t1[i] -= truemass[c]
            c = sister[c]
        if m1[i] <= 0 or t1[i] <= 0.0:
            raise ValueError(f"node {i}: non-positive own mass")
    # most massive sub (strict >, first in the sister chain wins), bottom-up (NEI:296-316)
    most = np.full(nn + 1, -1, np.int64)
    m2, t2 = m1.copy(), t1.copy()
    for i in range(nn, 0, -1):
        c = firstchild[i]
        if c > 0:
            best, mx = c, t2[c]
            c = sister[c]
            while c > 0:
                if t2[c] > mx:
                    best, mx = c, t2[c]
                c = sister[c]
            most[i] = best
            m2[i] += m2[best]
            t2[i] += t2[best]
    # structures (NEI:318-343)
    idx = np.arange(1, nn + 1)
    mo = mother[1:]
    is_halo = mo <= 0
    is_most = (~is_halo) & (idx == most[np.where(is_halo, 0, mo)])
    is_start = is_halo | ~is_most
    sid = np.zeros(nn + 1, np.int64)
    sid[1:][is_start] = np.cumsum(is_start)[is_start]
    parent = idx.copy()
    parent[is_most] = mo[is_most]
    par = np.zeros(nn + 1, np.int64)
    par[1:] = parent
    for _ in range(64):
        nxt = par[par]
        if np.array_equal(nxt, par):
            break
        par = nxt
    node_to_struct = sid[par]
    nstruct = int(is_start.sum())
    wp = np.asarray(liste_parts).copy()
    sel = wp > 0
    wp[sel] = node_to_struct[wp[sel]]
    # structure tree (NEI:399-425)
    mother_s = np.full(nstruct, -1, np.int64)
    first_sister = np.full(nstruct, -1, np.int64)
    first_daughter = np.full(nstruct, -1, np.int64)
    level_s = np.zeros(nstruct, np.int64)
    ihalo = -1
    for i in range(1, nn + 1):
        k = node_to_struct[i]
        if mother_s[k - 1] < 0:
            if mother[i] <= 0:
                mother_s[k - 1] = 0
                if ihalo > 0:
                    first_sister[ihalo - 1] = k
                ihalo = k
                level_s[k - 1] = 1
            else:
                m = node_to_struct[mother[i]]
                mother_s[k - 1] = m
                level_s[k - 1] = level_s[m - 1] + 1
                if first_daughter[m - 1] <= 0:
                    first_daughter[m - 1] = k
                else:
                    s = first_daughter[m - 1]
                    while first_sister[s - 1] > 0:
                        s = first_sister[s - 1]
                    first_sister[s - 1] = k
    return dict(whereIam_parts=wp, nstruct=nstruct, nb_of_halos=int(is_halo.sum()),
                nb_of_subhalos=int((~is_halo & ~is_most).sum()), mother=mother_s, first_sister=first_sister,
                first_daughter=first_daughter, level=level_s)


def group_members(whereIam_parts):
    """(order, unis, idxs, counts) with members of each structure contiguous."""
    order = np.argsort(whereIam_parts, kind="stable")
    unis, idxs, counts = np.unique(whereIam_parts[order], return_index=True, return_counts=True)
    return order, unis, idxs, counts
