"""Invariants of the oracle's particle advance in its three centers
(padvnc3d fullv, halfv and synchv, w3d.F:1862-2310), which the GPU advance
matches bit for bit in tests/test_gpu_particles.py:
- in a uniform E field with no lattice, fullv kicks by q E dt / m, halfv
  and synchv by half of that, and halfv followed by fullv steps keeps the
  velocity half a step ahead of the positions;
- inside a quad, the Boris rotation conserves |u| in every center;
- across a quad edge the kick scales with the residence fraction of the
  center's time window;
- synchv moves no particle and applies no boundary."""
import numpy as np
import pytest

from oracle import oracle
from warp_b200.constants import echarge, proton_mass


def _beam(n, seed=0):
    rng = np.random.default_rng(seed)
    return {"x": rng.normal(0, 2e-3, n), "y": rng.normal(0, 2e-3, n), "z": rng.uniform(0.3, 0.7, n),
            "ux": rng.normal(0, 1e4, n), "uy": rng.normal(0, 1e4, n), "uz": np.full(n, 1.4e7), "gaminv": np.ones(n)}


def _push(p, e, dt, center, tables=None, zlmin=0.0, dzl=1.0):
    n = len(p["x"])
    ex, ey, ez = (np.full(n, v) for v in e)
    oracle.push(p, ex, ey, ez, echarge, proton_mass, dt, tables, zlmin, dzl, 0.0, 1.0, 1.0, center=center)


@pytest.mark.parametrize("center,frac", [("fullv", 1.0), ("halfv", 0.5), ("synchv", 0.5)])
def test_uniform_field_kick(center, frac):
    p = _beam(1000)
    u0 = {k: p[k].copy() for k in ("ux", "uy", "uz")}
    e, dt = (2e4, -1e4, 5e3), 3e-10
    _push(p, e, dt, center)
    for k, ek in zip(("ux", "uy", "uz"), e):
        assert np.allclose(p[k] - u0[k], frac * echarge * ek * dt / proton_mass, rtol=1e-9, atol=1e-6)


def test_halfv_then_fullv_is_leapfrog():
    """A halfv step and fullv steps give x(t+n dt) of the exact
    uniform-acceleration motion, with the velocities at t + (n-1/2) dt."""
    p = _beam(200)
    x0, ux0 = p["x"].copy(), p["ux"].copy()
    e, dt, nsteps = (3e4, 0.0, 0.0), 2e-10, 5
    _push(p, e, dt, "halfv")
    for _ in range(nsteps - 1):
        _push(p, e, dt, "fullv")
    a = echarge * e[0] / proton_mass
    t = nsteps * dt
    assert np.allclose(p["x"], x0 + ux0 * t + 0.5 * a * t * t, rtol=1e-12, atol=1e-15)
    assert np.allclose(p["ux"], ux0 + a * (t - 0.5 * dt), rtol=1e-12)
    x = p["x"].copy()
    _push(p, e, dt, "synchv")
    assert np.array_equal(p["x"], x)
    assert np.allclose(p["ux"], ux0 + a * t, rtol=1e-12)


@pytest.mark.parametrize("center", ["fullv", "halfv", "synchv"])
def test_quad_rotation_conserves_speed(center):
    from warp_b200.lattice import fodo
    lat = fodo(40.0, 0.2, 0.5)
    nzl, zlmin, dzl = 64, 0.0, 1.0 / 64
    tables = lat.tables(zlmin, dzl, nzl)
    p = _beam(2000, seed=1)
    p["z"][:] = np.random.default_rng(2).uniform(0.0, 0.1, 2000)  # inside the focusing quad
    u2 = p["ux"] ** 2 + p["uy"] ** 2 + p["uz"] ** 2
    _push(p, (0.0, 0.0, 0.0), 2e-10, center, tables=tables[:3], zlmin=zlmin, dzl=dzl)
    assert np.allclose(p["ux"] ** 2 + p["uy"] ** 2 + p["uz"] ** 2, u2, rtol=1e-12)
    assert not np.allclose(p["ux"], _beam(2000, seed=1)["ux"])  # the quad did act


def test_synchv_applies_no_boundary():
    p = _beam(100)
    p["x"][:10] = 0.5  # outside a pipe of radius 0.01
    n = len(p["x"])
    z = np.zeros(n)
    oracle.push(p, z, z, z, echarge, proton_mass, 1e-10, None, 0.0, 1.0, 0.0, 1.0, 0.01, center="synchv")
    assert np.all(p["gaminv"] == 1.0)
    oracle.push(p, z, z, z, echarge, proton_mass, 1e-10, None, 0.0, 1.0, 0.0, 1.0, 0.01, center="fullv")
    assert np.all(p["gaminv"][:10] == 0.0)


@pytest.mark.parametrize("center,window", [("fullv", (-0.5, 0.5)), ("halfv", (0.0, 0.5)), ("synchv", (-0.5, 0.0))])
@pytest.mark.parametrize("side", ["entry", "exit"])
def test_quad_kick_scales_with_residence_fraction(center, window, side):
    """applyquad (top_lattice.F:2985-3120): a particle whose time window
    [z + vz dtl, z + vz dtr] straddles a quad edge feels the quad's field
    times the fraction of the window inside the quad. With a weak gradient
    the Boris kick is linear in the field, so the kick of a straddling
    particle is that fraction of the kick of one inside the quad."""
    from warp_b200.lattice import Lattice, Quad
    zs, ze, db = 0.40, 0.55, 1e-3
    lat = Lattice([Quad(zs, ze, db)], zlatperi=1.0)
    nzl, zlmin, dzl = 200, 0.0, 1.0 / 200
    tables = lat.tables(zlmin, dzl, nzl)[:3]
    dt, vz = 2e-9, 1.4e7
    a = vz * dt * (window[1] - window[0])
    f = np.array([0.1, 0.25, 0.5, 0.8, 0.97])
    n = len(f) + 1
    if side == "entry":  # window from zs - (1 - f) a to zs + f a
        zl = zs - (1.0 - f) * a
    else:  # window from ze - f a to ze + (1 - f) a
        zl = ze - f * a
    z = np.concatenate([zl - vz * dt * window[0], [0.5 * (zs + ze)]])
    p = {"x": np.full(n, 1e-3), "y": np.zeros(n), "z": z, "ux": np.zeros(n), "uy": np.zeros(n),
         "uz": np.full(n, vz), "gaminv": np.ones(n)}
    _push(p, (0.0, 0.0, 0.0), dt, center, tables=tables, zlmin=zlmin, dzl=dzl)
    kick = p["ux"][:-1] / p["ux"][-1]
    assert p["ux"][-1] != 0.0
    assert np.allclose(kick, f, rtol=1e-9, atol=0), kick
