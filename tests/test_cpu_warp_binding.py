"""The WARP-side binding's translation of WARP's conductor objects (by
class, from the attributes generateconductors.py sets) and its refusals."""
import pytest

from tests import warp_standins as W


def test_shapes_from_warp_conductors():
    from warp_b200.warp_binding import shape_from_warp
    pipe = W.ZCylinderOut(radius=0.45, zlower=-2.0, zupper=4.0)
    s = shape_from_warp(pipe)
    assert s.kind == 0 and s.radius == 0.45 and s.length == 6.0 and s.zcent == 1.0
    assert s.condid == pipe.condid
    rod = W.ZCylinder(radius=0.05, length=0.5, voltage=0.3, xcent=-0.1, ycent=-0.2, zcent=0.1)
    r = shape_from_warp(rod)
    assert (r.kind, r.length, r.voltage, r.xcent, r.ycent, r.zcent) == (1, 0.5, 0.3, -0.1, -0.2, 0.1)
    sph = W.Sphere(radius=0.12, voltage=0.7, xcent=0.15, condid=42)
    t = shape_from_warp(sph)
    assert (t.kind, t.radius, t.voltage, t.condid) == (2, 0.12, 0.7, 42)
    # condid='next' is WARP's counter: successive objects get successive ids
    a, b = W.Sphere(radius=0.1), W.Sphere(radius=0.1)
    assert shape_from_warp(b).condid == shape_from_warp(a).condid + 1


def test_unsupported_conductors_are_refused():
    from warp_b200.warp_binding import shape_from_warp
    with pytest.raises(NotImplementedError, match="Box"):
        shape_from_warp(W.Box(0.1, 0.1, 0.1))
    c = W.ZCylinderOut(radius=0.4, length=1.0)
    c.length = None
    with pytest.raises(ValueError):
        shape_from_warp(c)
