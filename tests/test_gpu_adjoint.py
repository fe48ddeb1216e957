"""Adjoint kernels vs FP64 central finite differences and direct-sum forces.

* SPHDensity: the fixed-list density reproduces the finder's density bit for
  bit with the finder's own lists; d(sum g*rho)/dx from the adjoint kernel
  matches central differences (h = 1e-7) on random particles to 1e-6 relative
  (of the largest gradient component in the sample).
* HaloPotential: dE/dx equals minus the direct-sum gravitational force
  (numpy, FP64) to 1e-10 and matches central differences of E to 1e-6.
"""
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


def test_density_adjoint_matches_finite_differences():
    import torch
    from ahop_b200 import autograd, finder, synthetic
    ps = synthetic.clustered_box(60000, 80, seed=44, nmax=4000)
    finder.configure(ps.n)
    st = finder.run_stages(ps.pos, ps.mass, last_stage=2, store_neighbours=32)
    nei = st["neighbours"] - 1  # 0-based, sorted by (distance, index)
    dev = torch.device("cuda:0")
    pos = torch.from_numpy(ps.pos.copy()).to(dev).requires_grad_(True)
    mass = torch.from_numpy(ps.mass).to(dev)
    nei_t = torch.from_numpy(np.ascontiguousarray(nei, np.int32)).to(dev)
    rho = autograd.SPHDensity.apply(pos, mass, nei_t, 1.0)
    assert np.array_equal(rho.detach().cpu().numpy(), st["density"])  # same bits as the finder
    rng = np.random.default_rng(1)
    g = torch.from_numpy(rng.normal(size=ps.n)).to(dev)
    (rho * g).sum().backward()
    grad = pos.grad.cpu().numpy()
    # particles whose density depends on particle j: j itself and every i listing j
    users = [[] for _ in range(ps.n)]
    for i in range(ps.n):
        for j in nei[i]:
            users[j].append(i)
    h = 1e-7
    gn = g.cpu().numpy()
    sample = rng.choice(ps.n, 60, replace=False)
    fd = np.zeros((len(sample), 3))
    for a, j in enumerate(sample):
        aff = np.array(sorted(set(users[j] + [j])))
        for ax in range(3):
            vals = []
            for sgn in (+1, -1):
                p = ps.pos.copy()
                p[j, ax] += sgn * h
                r = autograd.density_fixed(torch.from_numpy(p).to(dev), mass, nei_t, 1.0).cpu().numpy()
                vals.append(np.dot(gn[aff], r[aff]))
            fd[a, ax] = (vals[0] - vals[1]) / (2 * h)
    adj = grad[sample]
    scale = np.abs(fd).max()
    assert np.abs(adj - fd).max() <= 1e-6 * scale, np.abs(adj - fd).max() / scale


def _forces(off, pos, mass, L, G):
    f = np.zeros_like(pos)
    for h in range(len(off) - 1):
        a, b = off[h], off[h + 1]
        p = pos[a:b]
        d = p[:, None, :] - p[None, :, :]
        d[d > L / 2] -= L
        d[d < -L / 2] += L
        r2 = (d * d).sum(-1)
        np.fill_diagonal(r2, np.inf)
        f[a:b] = -G * mass[a:b, None] * (mass[None, a:b, None] * d / r2[..., None] ** 1.5).sum(1)
    return f


def test_potential_gradient_is_minus_direct_force():
    import torch
    from ahop_b200 import autograd, synthetic
    off, pos, vel, mass, dens = synthetic.halo_catalogue(40, seed=5, nmin=20, nmax=1500, box=100.0)
    G = 430.1
    dev = torch.device("cuda:0")
    p = torch.from_numpy(pos.copy()).to(dev).requires_grad_(True)
    m = torch.from_numpy(mass).to(dev)
    off_t = torch.from_numpy(off)
    ep = autograd.HaloPotential.apply(p, m, off_t, 100.0, G)
    gh = torch.ones_like(ep)
    (ep * gh).sum().backward()
    grad = p.grad.cpu().numpy()
    F = _forces(off, pos, mass, 100.0, G)
    np.testing.assert_allclose(grad, -F, rtol=1e-10, atol=1e-12 * np.abs(F).max())
    # central differences of E on a few particles
    h = 1e-7
    rng = np.random.default_rng(2)
    for j in rng.choice(off[-1], 10, replace=False):
        hh = np.searchsorted(off, j, side="right") - 1
        for ax in range(3):
            vals = []
            for sgn in (+1, -1):
                q = pos.copy()
                q[j, ax] += sgn * h
                e = autograd.HaloPotential.apply(torch.from_numpy(q).to(dev), m, off_t, 100.0, G)
                vals.append(float(e[hh]))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(fd - grad[j, ax]) <= 1e-6 * max(abs(grad[j, ax]), np.abs(F[off[hh]:off[hh + 1]]).max())
