"""Edge cases of the PIC step on the GPU:
- empty and fully lost particle groups;
- particles exactly on the upper grid faces (against the oracle);
- zero charge;
- the smallest grid (against the oracle);
- non-convergence within mgmaxiters;
- the error codes for a non-finite rho, for the fixed-point accumulator
  overflow, and for bad or too large grids.
"""
import numpy as np
import pytest
import torch

from oracle import oracle
from tests import gpu_helpers as H

pytestmark = pytest.mark.gpu


def _solver(nx=16, ny=16, nz=32, bounds=(0, 0, 0, 0, 2, 2), **kw):
    return H.make_solver(nx, ny, nz, (-0.04, -0.04, 0.0), (0.04, 0.04, 1.0), bounds, **kw)


def _group(p, w=1e4):
    from warp_b200.particles import ParticleGroup
    return ParticleGroup(p, w=w)


def _beam(n, seed=1):
    from warp_b200.particles import semigaussian
    return semigaussian(n, seed=seed, radius=4e-3)


def test_empty_particle_group():
    s = _solver()
    pg = _group({k: np.zeros(0) for k in ("x", "y", "z", "ux", "uy", "uz", "gaminv")})
    s.loadrho(pgroups=[pg])
    assert float(s.rho.abs().max()) == 0.0
    s.advance(pg, 1e-9)
    s.fetche(pg)
    assert s.moments(pg)["n"] == 0
    pg.sort(s)
    assert pg.np == 0


def test_all_particles_lost():
    s = _solver()
    p = _beam(5000)
    p["gaminv"][:] = 0.0
    pg = _group(p)
    s.loadrho(pgroups=[pg])
    assert float(s.rho.abs().max()) == 0.0
    x0 = pg.x.clone()
    s.advance(pg, 1e-9)
    assert torch.equal(pg.x, x0)
    assert s.moments(pg)["n"] == 0
    pg.sort(s)
    assert pg.np == 0


def test_particles_on_upper_faces_match_oracle():
    """Particles exactly on x = xmax, y = ymax, z = zmax deposit into the last
    cell with fraction 1 and gather from it, as the oracle does."""
    s = _solver()
    n = 64
    rng = np.random.default_rng(3)
    p = {"x": rng.uniform(-0.04, 0.04, n), "y": rng.uniform(-0.04, 0.04, n), "z": rng.uniform(0.0, 1.0, n),
         "ux": np.zeros(n), "uy": np.zeros(n), "uz": np.zeros(n), "gaminv": np.ones(n)}
    p["x"][::3] = 0.04
    p["y"][1::3] = 0.04
    p["z"][2::3] = 1.0
    p["x"][0], p["y"][0], p["z"][0] = 0.04, 0.04, 1.0
    pg = _group(p)
    s.loadrho(pgroups=[pg], lfinalize_rho=False)
    ref = np.zeros((s.nx + 1, s.ny + 1, s.nz + 1), order="F")
    oracle.setrho(ref, p["x"], p["y"], p["z"], pg.q, pg.w, s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin,
                  gaminv=p["gaminv"])
    got = s.rho.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
    phi = np.asfortranarray(rng.standard_normal((s.nx + 3, s.ny + 3, s.nz + 3)))
    s.phi = phi
    s.fetche(pg)
    ex, ey, ez = oracle.sete(phi, p["x"], p["y"], p["z"], s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin)
    assert np.array_equal(pg.ex.cpu().numpy(), ex)
    assert np.array_equal(pg.ey.cpu().numpy(), ey)
    assert np.array_equal(pg.ez.cpu().numpy(), ez)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_zero_charge_gives_conductor_potentials(precision):
    from warp_b200 import conductors as C
    s = _solver(tolkind="relres", mgtol=1e-9, precision=precision)
    s.installconductor(C.ZCylinder(radius=0.01, length=10.0, voltage=2.0, zcent=0.5))
    s.rho = np.zeros((s.nx + 1, s.ny + 1, s.nz + 1))
    s.solve()
    assert s.converged
    phi = s.phi.cpu().numpy()
    assert np.isfinite(phi).all()
    assert 0.0 < phi.max() <= 2.0 + 1e-12
    s.clearconductors()
    s.phi = np.zeros_like(phi)
    s.solve()
    assert float(s.phi.abs().max()) == 0.0


def test_smallest_grid_matches_oracle():
    s = H.make_solver(2, 2, 2, (0., 0., 0.), (1., 1., 1.), (1, 1, 0, 0, 2, 2), mgtol=1e-12)
    rho = np.asfortranarray(np.random.default_rng(5).standard_normal((3, 3, 3))) * 1e-9
    s.rho = rho
    s.solve()
    ref = np.zeros((5, 5, 5), order="F")
    oracle.mgsolve(ref, rho, 1.0 / 2, 1.0 / 2, 1.0 / 2, (1, 1, 0, 0, 2, 2), mgtol=1e-12)
    assert np.array_equal(s.phi.cpu().numpy(), ref)


def test_not_converged_within_mgmaxiters():
    s = _solver(tolkind="relres", mgtol=1e-14, mgmaxiters=1)
    s.rho = H.gaussian_blobs_rho(s.nx, s.ny, s.nz, (s.xmmin, s.ymmin, s.zmmin), (s.xmmax, s.ymmax, s.zmmax), 3, 2,
                                 oracle.eps0())
    s.solve()
    assert s.mgiters == 1
    assert not s.converged


def test_nonfinite_rho_is_rejected():
    from warp_b200._lib import WgError
    s = _solver()
    rho = np.zeros((s.nx + 1, s.ny + 1, s.nz + 1))
    rho[3, 4, 5] = np.nan
    s.rho = rho
    with pytest.raises(WgError, match="NaN or Inf"):
        s.solve()


def test_accumulator_overflow_is_reported():
    """70000 full particle weights on one node pass 2^62 in the fixed-point
    accumulator: the deposit reports WG_EOVERFLOW instead of wrapping."""
    from warp_b200._lib import WgError
    s = _solver()
    n = 70000
    x0, y0, z0 = s.xmmin + 5 * s.dx, s.ymmin + 5 * s.dy, s.zmmin + 5 * s.dz
    p = {"x": np.full(n, x0), "y": np.full(n, y0), "z": np.full(n, z0), "ux": np.zeros(n), "uy": np.zeros(n),
         "uz": np.zeros(n), "gaminv": np.ones(n)}
    pg = _group(p)
    with pytest.raises(WgError) as e:
        s.loadrho(pgroups=[pg])
    assert e.value.code == -4


def test_chunked_deposit_matches_loadrho_and_checks_its_use():
    from warp_b200._lib import WgError
    s = _solver()
    p = _beam(30_000, seed=4)
    pg = _group(p)
    s.loadrho(pgroups=[pg])
    ref = s.rho.clone()
    s.deposit_begin()
    for a, b in ((0, 7000), (7000, 7000), (7000, 30_000)):
        s.deposit_add(pg, a, b)
    s.deposit_end()
    assert torch.equal(s.rho, ref)
    # pieces with another weight, a plain deposit while open, add after end
    s.deposit_begin()
    s.deposit_add(pg, 0, 100)
    with pytest.raises(WgError) as e:
        s.deposit_add(_group(p, w=2e4), 100, 200)
    assert e.value.code == -1
    with pytest.raises(WgError) as e:
        s.loadrho(pgroups=[pg])
    assert e.value.code == -3
    s.deposit_end()
    with pytest.raises(WgError) as e:
        s.deposit_add(pg, 0, 10)
    assert e.value.code == -3


def test_chunked_deposit_overflow_is_reported_by_the_next_solve():
    from warp_b200._lib import WgError
    s = _solver()
    n = 70000
    x0, y0, z0 = s.xmmin + 5 * s.dx, s.ymmin + 5 * s.dy, s.zmmin + 5 * s.dz
    p = {"x": np.full(n, x0), "y": np.full(n, y0), "z": np.full(n, z0), "ux": np.zeros(n), "uy": np.zeros(n),
         "uz": np.zeros(n), "gaminv": np.ones(n)}
    pg = _group(p)
    s.deposit_begin()
    s.deposit_add(pg, 0, 40000)
    s.deposit_add(pg, 40000, n)
    s.deposit_end()
    with pytest.raises(WgError) as e:
        s.solve()
    assert e.value.code == -4
    # the flag is cleared once reported
    s.rho = np.zeros((s.nx + 1, s.ny + 1, s.nz + 1))
    s.solve()


def test_bad_and_too_large_grids():
    from warp_b200._lib import WgError
    with pytest.raises(WgError) as e:
        H.make_solver(1, 8, 8, (0., 0., 0.), (1., 1., 1.), (0,) * 6)
    assert e.value.code == -1
    with pytest.raises(WgError) as e:
        H.make_solver(8, 8, 8, (0., 0., 0.), (1., 1., 1.), (0, 0, 0, 0, 2, 0))
    assert e.value.code == -1
    with pytest.raises(WgError) as e:
        H.make_solver(2048, 2048, 1024, (0., 0., 0.), (1., 1., 1.), (0,) * 6)
    assert e.value.code == -7
