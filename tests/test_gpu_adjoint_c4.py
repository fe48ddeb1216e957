"""Differentiation at its full stated configuration: 2,097,152 particles in
2,000 NFW halos of up to ~74,000 members (the c4_2m workload, seed 4).

* SPH density with the finder's 32-neighbour lists held fixed: the
  fixed-list density equals the finder's bit for bit; d(sum g rho)/dx from
  the adjoint kernel matches FP64 central differences (h = 1e-7) on 1,000
  random particles to 1e-6 relative (of the largest gradient component in
  the sample).
* Per-halo direct-sum potential over the generator's halos: dE/dx equals
  minus the direct-sum force (NumPy FP64, per sampled particle over its
  halo) to 1e-10 on 1,000 random halo members, and matches FP64 central
  differences of E to 1e-6 of the halo's largest gradient component plus the
  differences' own truncation bound: a directional third derivative of 1/r is
  at most 6/r^4, so |fd - dE/dx| <= h^2 G m_j sum_i m_i / (r_ij - h)^4 (this
  matters for members with a neighbour closer than ~100 h).  E
  depends on x_j only through the pairs (i, j), so the differences are taken
  of those n - 1 terms (NumPy FP64); for halos of up to 5,000 members they
  are also taken of the whole E through the forward kernel.  For larger
  halos the kernel's E is a sum of up to 2.8e9 pair terms whose FP64
  rounding, divided by 2h, exceeds 1e-6 of the gradient (measured: 3.6e-5
  relative in the largest halo), so there only the pair-term differences
  apply.
The backward passes recompute the pair weights from positions; nothing is
stored between forward and backward but positions and lists.
"""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

H = 1e-7
NSAMPLE = 1000


@pytest.fixture(scope="module")
def c4():
    if not gpu_available():
        pytest.skip("no CUDA device")
    from ahop_b200 import build, finder, synthetic
    build.build()
    ps = synthetic.workload("c4_2m")
    assert ps.n == 2_097_152 and len(ps.halo_counts) == 2000
    finder.configure(ps.n)
    st = finder.run_stages(ps.pos, ps.mass, last_stage=2, store_neighbours=32)
    return ps, st


def test_density_adjoint_c4(c4):
    import torch
    from ahop_b200 import autograd
    ps, st = c4
    dev = torch.device("cuda:0")
    nei = torch.from_numpy(np.ascontiguousarray(st["neighbours"] - 1, np.int32)).to(dev)
    pos0 = torch.from_numpy(ps.pos.copy()).to(dev)
    mass = torch.from_numpy(ps.mass).to(dev)
    pos = pos0.clone().requires_grad_(True)
    rho = autograd.SPHDensity.apply(pos, mass, nei, 1.0)
    assert np.array_equal(rho.detach().cpu().numpy(), st["density"])
    rng = np.random.default_rng(4)
    g = torch.from_numpy(rng.normal(size=ps.n)).to(dev)
    (rho * g).sum().backward()
    grad = pos.grad.cpu().numpy()
    sample = rng.choice(ps.n, NSAMPLE, replace=False)
    fd = np.zeros((NSAMPLE, 3))
    work = pos0.clone()
    ids = torch.arange(ps.n, device=dev)
    for a, j in enumerate(sample):
        aff = ((nei == int(j)).any(1) | (ids == int(j))).nonzero().squeeze(1)
        for ax in range(3):
            vals = []
            for sgn in (+1, -1):
                work[j, ax] = pos0[j, ax] + sgn * H
                r = autograd.density_fixed(work, mass, nei, 1.0)
                vals.append(float((g[aff] * r[aff]).sum()))
            work[j, ax] = pos0[j, ax]
            fd[a, ax] = (vals[0] - vals[1]) / (2 * H)
    adj = grad[sample]
    scale = np.abs(fd).max()
    assert np.abs(adj - fd).max() <= 1e-6 * scale, np.abs(adj - fd).max() / scale


def test_potential_adjoint_c4(c4):
    import torch
    from ahop_b200 import autograd, halo_props
    ps, _ = c4
    G, L = 430.1, 1.0
    dev = torch.device("cuda:0")
    order = np.argsort(ps.halo_id, kind="stable")
    order = order[ps.halo_id[order] >= 0]
    counts = np.bincount(ps.halo_id[order])
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    hp = np.ascontiguousarray(ps.pos[order])
    hm = np.ascontiguousarray(ps.mass[order])
    m_t = torch.from_numpy(hm).to(dev)
    p = torch.from_numpy(hp.copy()).to(dev).requires_grad_(True)
    ep = autograd.HaloPotential.apply(p, m_t, torch.from_numpy(off), L, G)
    ep.sum().backward()
    grad = p.grad.cpu().numpy()
    rng = np.random.default_rng(5)
    sample = np.sort(rng.choice(off[-1], NSAMPLE, replace=False))
    halo = np.searchsorted(off, sample, side="right") - 1
    # minus the direct-sum force on each sampled member, over its own halo
    for j, hh in zip(sample, halo):
        a, b = off[hh], off[hh + 1]
        d = hp[j] - hp[a:b]
        d[d > L / 2] -= L
        d[d < -L / 2] += L
        r2 = (d * d).sum(1)
        r2[j - a] = np.inf
        f = -G * hm[j] * (hm[a:b, None] * d / r2[:, None] ** 1.5).sum(0)
        np.testing.assert_allclose(grad[j], -f, rtol=1e-10, atol=1e-12 * np.abs(f).max())
    # central differences of the pair terms of each sampled member
    def separations(x, j, a, b):
        d = x - hp[a:b]
        d[d > L / 2] -= L
        d[d < -L / 2] += L
        r = np.sqrt((d * d).sum(1))
        r[j - a] = np.inf
        return r

    def pair_energy(x, j, a, b):
        return -G * hm[j] * np.sum(hm[a:b] / separations(x, j, a, b))

    trunc = {}
    for j, hh in zip(sample, halo):
        a, b = off[hh], off[hh + 1]
        trunc[j] = H * H * G * hm[j] * np.sum(hm[a:b] / (separations(hp[j], j, a, b) - H) ** 4)
        gmax = np.abs(grad[a:b]).max()
        for ax in range(3):
            e = np.zeros(3)
            e[ax] = H
            fdv = (pair_energy(hp[j] + e, j, a, b) - pair_energy(hp[j] - e, j, a, b)) / (2 * H)
            assert abs(fdv - grad[j, ax]) <= 1e-6 * max(abs(grad[j, ax]), gmax) + trunc[j], (j, ax)
    # central differences of the halo's E through the forward kernel
    halo_props.set_graph(False)
    try:
        for hh in np.unique(halo):
            a, b = off[hh], off[hh + 1]
            if b - a > 5000:
                continue
            q0 = torch.from_numpy(hp[a:b].copy()).to(dev)
            q = q0.clone()
            mh = m_t[a:b]
            o1 = torch.tensor([0, b - a], dtype=torch.int64)
            gmax = np.abs(grad[a:b]).max()
            for j in sample[halo == hh]:
                for ax in range(3):
                    vals = []
                    for sgn in (+1, -1):
                        q[j - a, ax] = q0[j - a, ax] + sgn * H
                        vals.append(float(autograd.HaloPotential.apply(q, mh, o1, L, G)[0]))
                    q[j - a, ax] = q0[j - a, ax]
                    fdv = (vals[0] - vals[1]) / (2 * H)
                    assert abs(fdv - grad[j, ax]) <= 1e-6 * max(abs(grad[j, ax]), gmax) + trunc[j], (j, ax)
    finally:
        halo_props.set_graph(True)
