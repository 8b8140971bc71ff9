"""Invariants of the oracle's CIC deposit (setrho3ddirect1,
w3d.F:7757-7960; rho boundary fold, w3d.F:2660-2750) and field gather
(sete_from_phi_linear3d, w3d.F:3963-4196), which pin both beyond the
restatement:
- the deposited charge is q w per particle, and the first moments of rho
  are the particles' (linear weighting keeps them);
- a particle on a node puts all its charge there, one at a cell centre an
  eighth on each corner;
- deposit is additive over particle sets;
- a linear phi gives the exact uniform E anywhere in the grid;
- gather and deposit use the same weights: the sum over particles of the
  gathered E equals the sum over nodes of (rho / g) times the node E.
The product's deposit and gather match the oracle on the GPU
(tests/test_gpu_particles.py)."""
import numpy as np
import pytest

from oracle import oracle

NX, NY, NZ = 12, 10, 16
MINS = (-0.03, -0.02, 0.1)
D = (0.005, 0.004, 0.025)
Q, W = 1.6e-19, 3.5e4


def _beam(n, seed, margin=0.0):
    rng = np.random.default_rng(seed)
    lo = [MINS[k] + margin * D[k] for k in range(3)]
    hi = [MINS[k] + (N - margin) * D[k] for k, N in enumerate((NX, NY, NZ))]
    return [rng.uniform(lo[k], hi[k], n) for k in range(3)]


def _rho(x, y, z):
    rho = np.zeros((NX + 1, NY + 1, NZ + 1), order="F")
    oracle.setrho(rho, x, y, z, Q, W, *D, *MINS)
    return rho


def _nodes():
    return np.meshgrid(*(MINS[k] + np.arange(n + 1) * D[k] for k, n in enumerate((NX, NY, NZ))), indexing="ij")


def test_charge_and_first_moments_are_kept():
    x, y, z = _beam(5000, 1)
    rho = _rho(x, y, z)
    dv = D[0] * D[1] * D[2]
    total = Q * W * len(x)
    assert rho.sum() * dv == pytest.approx(total, rel=1e-13)
    gx, gy, gz = _nodes()
    for g, p in ((gx, x), (gy, y), (gz, z)):
        assert (rho * g).sum() * dv == pytest.approx(Q * W * p.sum(), rel=1e-12)
    # the periodic fold keeps the charge on the nodes 0..nz-1
    oracle.rhobc(rho, (0, 0, 0, 0, 2, 2))
    assert np.array_equal(rho[:, :, 0], rho[:, :, NZ])
    assert rho[:, :, :NZ].sum() * dv == pytest.approx(total, rel=1e-13)


def test_node_and_cell_centre_weights():
    g = Q * W / (D[0] * D[1] * D[2])
    i, j, k = 3, 4, 5
    p = [np.array([MINS[a] + idx * D[a]]) for a, idx in enumerate((i, j, k))]
    rho = _rho(*p)
    assert rho[i, j, k] == pytest.approx(g, rel=1e-14)
    rest = rho.copy()
    rest[i, j, k] = 0.0
    assert np.abs(rest).max() <= 1e-14 * g
    c = [np.array([MINS[a] + (idx + 0.5) * D[a]]) for a, idx in enumerate((i, j, k))]
    rho = _rho(*c)
    corners = rho[i:i + 2, j:j + 2, k:k + 2]
    assert np.allclose(corners, g / 8, rtol=1e-14)
    assert rho.sum() == pytest.approx(g, rel=1e-14)


def test_deposit_is_additive():
    a = _beam(3000, 2)
    b = _beam(2000, 3)
    both = [np.concatenate([a[k], b[k]]) for k in range(3)]
    ra, rb, rab = _rho(*a), _rho(*b), _rho(*both)
    assert np.max(np.abs(rab - (ra + rb))) <= 1e-13 * np.max(np.abs(rab))


def test_linear_phi_gives_exact_uniform_field():
    ca, cb, cc = 120.0, -75.0, 40.0
    ix = MINS[0] + (np.arange(NX + 3) - 1) * D[0]
    iy = MINS[1] + (np.arange(NY + 3) - 1) * D[1]
    iz = MINS[2] + (np.arange(NZ + 3) - 1) * D[2]
    X, Y, Z = np.meshgrid(ix, iy, iz, indexing="ij")
    phi = np.asfortranarray(ca * X + cb * Y + cc * Z + 3.0)
    x, y, z = _beam(4000, 4)
    ex, ey, ez = oracle.sete(phi, x, y, z, *D, *MINS)
    assert np.allclose(ex, -ca, rtol=1e-11, atol=0)
    assert np.allclose(ey, -cb, rtol=1e-11, atol=0)
    assert np.allclose(ez, -cc, rtol=1e-11, atol=0)


def test_gather_uses_the_deposit_weights():
    rng = np.random.default_rng(5)
    phi = np.asfortranarray(rng.standard_normal((NX + 3, NY + 3, NZ + 3)))
    x, y, z = _beam(3000, 6)
    ex, ey, ez = oracle.sete(phi, x, y, z, *D, *MINS)
    # node fields by centred differences (the gather's node values)
    enode = (-(phi[2:, 1:-1, 1:-1] - phi[:-2, 1:-1, 1:-1]) / (2 * D[0]),
             -(phi[1:-1, 2:, 1:-1] - phi[1:-1, :-2, 1:-1]) / (2 * D[1]),
             -(phi[1:-1, 1:-1, 2:] - phi[1:-1, 1:-1, :-2]) / (2 * D[2]))
    weights = _rho(x, y, z) / (Q * W / (D[0] * D[1] * D[2]))
    for eg, en in zip((ex, ey, ez), enode):
        scale = np.abs(eg).sum()
        assert eg.sum() == pytest.approx((weights * en).sum(), abs=1e-12 * scale)
