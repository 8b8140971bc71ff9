"""The oracle's conductor data checked against the shapes' geometry on every
multigrid level (conductordelfromintercepts, f3d_conductors.F:12-729; the
intercepts of ZCylinderOut, ZCylinder and Sphere; checkconductors,
f3d_mgrid.F:3964-4326):
- every finite del of a subgrid point, measured from the node along its
  axis in units of that level's cell, ends on the conductor surface, and the
  volt in that direction is the conductor's voltage;
- subgrid points lie outside the conductor and interior points inside;
- on every level, a node outside the conductor whose axis neighbour is
  inside is a subgrid point with a del of at most one cell toward that
  neighbour.
The product's lists equal the oracle's (tests/test_gpu_mg.py), so this pins
both by geometry rather than by restatement alone."""
import numpy as np
import pytest

from oracle import oracle

N = (24, 20, 28)
MINS = (-0.5, -0.45, -0.6)
MAXS = (0.5, 0.55, 0.6)
TOL = 1e-12
BIG = 1e30

SHAPES = {
    # kind, radius, length, voltage, centre
    "sphere": ("Sphere", 0.21, 0.0, 0.7, (0.03, -0.02, 0.01)),
    "rod": ("ZCylinder", 0.12, 0.5, -0.4, (-0.05, 0.07, 0.02)),
    "pipe": ("ZCylinderOut", 0.41, 10.0, 0.25, (0.01, 0.04, 0.0)),
}


def _inside(kind, radius, length, c, p):
    """Signed distance-like function: negative inside the conductor, zero on
    its surface, positive outside."""
    x, y, z = p[..., 0] - c[0], p[..., 1] - c[1], p[..., 2] - c[2]
    if kind == "Sphere":
        return np.sqrt(x * x + y * y + z * z) - radius
    r = np.sqrt(x * x + y * y)
    if kind == "ZCylinder":
        return np.maximum(r - radius, np.abs(z) - 0.5 * length)
    return radius - r  # ZCylinderOut: the conductor is outside the radius


def _case(name):
    kind, radius, length, volt, c = SHAPES[name]
    d = tuple((MAXS[k] - MINS[k]) / N[k] for k in range(3))
    oc = oracle.Conductors(*N, *d, *MINS)
    oc.add_shape(kind, radius, length, volt, *c)
    oc.finalize()
    return kind, radius, length, volt, c, oracle.mglevels(*N, *d), oc.export()


@pytest.mark.parametrize("name", sorted(SHAPES))
def test_dels_end_on_the_surface_with_the_conductor_voltage(name):
    kind, radius, length, volt, c, levels, e = _case(name)
    si, sd, sv, sl = e["subgrid"]
    assert len(sl) > 0
    checked = 0
    for lev, (n, h) in enumerate(levels):
        sel = sl == lev
        node = np.asarray(MINS) + si[sel] * np.asarray(h)
        f = _inside(kind, radius, length, c, node)
        assert np.all(f > -TOL), "subgrid point inside the conductor on level %d" % lev
        for k in range(6):
            axis, sign = k // 2, (-1.0 if k % 2 == 0 else 1.0)
            dk = sd[sel, k]
            fin = dk < BIG
            p = node[fin].copy()
            p[:, axis] += sign * dk[fin] * h[axis]
            assert np.all(np.abs(_inside(kind, radius, length, c, p)) <= TOL * 10), (lev, k)
            assert np.all(sv[sel, k][fin] == volt), (lev, k)
            assert np.all(dk[fin] >= 0.0)
            checked += int(fin.sum())
    assert checked > 0


@pytest.mark.parametrize("name", sorted(SHAPES))
def test_interior_points_inside_and_every_crossing_has_a_subgrid_point(name):
    kind, radius, length, volt, c, levels, e = _case(name)
    ii, iv, il = e["interior"]
    si, sd, sv, sl = e["subgrid"]
    for lev, (n, h) in enumerate(levels):
        sel = il == lev
        f = _inside(kind, radius, length, c, np.asarray(MINS) + ii[sel] * np.asarray(h))
        assert np.all(f <= TOL), "interior point outside the conductor on level %d" % lev
        assert np.all(iv[sel] == volt)
        # nodes of the level and their inside/outside state
        g = np.stack(np.meshgrid(*(MINS[k] + np.arange(n[k] + 1) * h[k] for k in range(3)), indexing="ij"), -1)
        fin = _inside(kind, radius, length, c, g)
        subs = {tuple(p): row for p, row in zip(map(tuple, si[sl == lev]), sd[sl == lev])}
        missing = 0
        for k in range(6):
            axis, step = k // 2, (-1 if k % 2 == 0 else 1)
            nb = np.roll(fin, -step, axis=axis)
            valid = np.ones(fin.shape, bool)
            idx = [slice(None)] * 3
            idx[axis] = 0 if step < 0 else -1
            valid[tuple(idx)] = False
            # outside node, neighbour clearly inside (not within rounding of the surface)
            cross = valid & (fin > TOL) & (nb < -1e-9)
            for p in zip(*np.nonzero(cross)):
                row = subs.get(tuple(int(v) for v in p))
                if row is None or not row[k] <= 1.0:
                    missing += 1
        assert missing == 0, "%d crossings without a subgrid del on level %d" % (missing, lev)
