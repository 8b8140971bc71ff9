"""lcorrectede on the B200 against the oracle, bit for bit: the gather next
to conductors from the subgrid data (sete3dwithconductor, efetch = 1,
f3d_mgrid.F:4774-5220), alone (fetche) and fused into the particle advance.
The conductors are a grounded pipe and a rod at 1 kV, so the cells hold
even and odd subgrid points and interior nodes; the particles cover the
rod's surface, the pipe's, the vacuum between, the grid's upper faces and
points outside the grid."""
import numpy as np
import pytest
import torch

from oracle import oracle
from tests import gpu_helpers as H

pytestmark = pytest.mark.gpu

NX, NY, NZ = 32, 32, 16
MINS, MAXS = (-0.04, -0.04, 0.0), (0.04, 0.04, 0.16)


def _setup(precision="fp64"):
    from warp_b200 import conductors as C
    s = H.make_solver(NX, NY, NZ, MINS, MAXS, (0, 0, 0, 0, 2, 2), mgtol=1e-11, precision=precision)
    shapes = [C.ZCylinderOut(radius=0.035, length=10.0, zcent=0.08),
              C.ZCylinder(radius=0.011, length=10.0, voltage=1000.0, xcent=0.003, ycent=-0.002, zcent=0.08)]
    for sh in shapes:
        s.installconductor(sh)
    rng = np.random.default_rng(21)
    s.rho = 1e-9 * rng.standard_normal((NX + 1, NY + 1, NZ + 1))
    s.solve()
    return s, shapes


def _particles(n, seed=4):
    rng = np.random.default_rng(seed)
    r = rng.uniform(0.0, 0.039, n)
    th = rng.uniform(0, 2 * np.pi, n)
    p = {"x": r * np.cos(th), "y": r * np.sin(th), "z": rng.uniform(0.0, 0.16, n),
         "ux": rng.normal(0, 1e4, n), "uy": rng.normal(0, 1e4, n), "uz": np.full(n, 1.4e7), "gaminv": np.ones(n)}
    # upper faces and points outside the grid
    p["x"][:20] = 0.04
    p["y"][20:40] = 0.04
    p["z"][40:60] = 0.16
    p["x"][60:70] = 0.0405
    p["z"][70:80] = -1e-4
    return p


def test_fetche_with_lcorrectede_matches_oracle():
    s, shapes = _setup()
    oc = H.oracle_conductors(s, shapes)
    p = _particles(60_000)
    from warp_b200.particles import ParticleGroup
    pg = ParticleGroup(p, w=1.0)
    s.lcorrectede = True
    s.fetche(pg)
    phi = s.phi.cpu().numpy()
    ex, ey, ez = oracle.sete_cond(oc, phi, p["x"], p["y"], p["z"], s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin)
    assert np.array_equal(pg.ex.cpu().numpy(), ex)
    assert np.array_equal(pg.ey.cpu().numpy(), ey)
    assert np.array_equal(pg.ez.cpu().numpy(), ez)
    # the correction changes the field next to the rod and nowhere far from it
    s.lcorrectede = False
    s.fetche(pg)
    plain = pg.ex.cpu().numpy()
    assert np.sum(plain != ex) > 100
    r2 = (p["x"] - 0.003) ** 2 + (p["y"] + 0.002) ** 2
    far = (r2 > (0.011 + 4 * s.dx) ** 2) & (r2 < (0.035 - 4 * s.dx) ** 2) & (np.arange(len(r2)) >= 80)
    assert np.allclose(plain[far], ex[far], rtol=1e-12, atol=1e-9 * np.abs(ex).max())
    # the host-array form
    s.lcorrectede = True
    eh = s.fetche_host(p["x"], p["y"], p["z"])
    assert np.array_equal(eh[0], ex) and np.array_equal(eh[1], ey) and np.array_equal(eh[2], ez)


@pytest.mark.parametrize("center", ["halfv", "fullv", "synchv"])
def test_advance_with_lcorrectede_matches_oracle(center):
    from warp_b200.particles import ParticleGroup
    s, shapes = _setup()
    oc = H.oracle_conductors(s, shapes)
    p = _particles(40_000, seed=5)
    pg = ParticleGroup({k: v.copy() for k, v in p.items()}, w=1.0)
    s.lcorrectede = True
    dt = 2e-10
    for _ in range(2):
        phi = s.phi.cpu().numpy()
        ex, ey, ez = oracle.sete_cond(oc, phi, p["x"], p["y"], p["z"], s.dx, s.dy, s.dz, s.xmmin, s.ymmin,
                                      s.zmmin)
        oracle.push(p, ex, ey, ez, pg.q, pg.m, dt, None, 0.0, 1.0, s.zmmin, s.zmmax, 0.035, center=center)
        s.advance(pg, dt, prwall=0.035, center=center)
        got = pg.to_numpy()
        for k in ("x", "y", "z", "ux", "uy", "uz", "gaminv"):
            assert np.array_equal(got[k], p[k]), k


def test_lcorrectede_follows_conductor_changes():
    """After the conductors change, the next corrected gather uses the new
    ones (icgrid and the point fields are rebuilt)."""
    from warp_b200 import conductors as C
    from warp_b200.particles import ParticleGroup
    s, shapes = _setup()
    s.lcorrectede = True
    p = _particles(20_000, seed=6)
    pg = ParticleGroup(p, w=1.0)
    s.fetche(pg)
    s.uninstallconductor(shapes[1])
    rod = C.Sphere(radius=0.012, voltage=-500.0, zcent=0.08)
    s.installconductor(rod)
    s.solve()
    s.fetche(pg)
    oc = H.oracle_conductors(s, [shapes[0], rod])
    ex, ey, ez = oracle.sete_cond(oc, s.phi.cpu().numpy(), p["x"], p["y"], p["z"], s.dx, s.dy, s.dz, s.xmmin,
                                  s.ymmin, s.zmmin)
    assert np.array_equal(pg.ex.cpu().numpy(), ex)
    assert np.array_equal(pg.ez.cpu().numpy(), ez)
