"""Conductor shapes for installconductor (the subset of
scripts/generateconductors.py used by the 3D ES PIC workloads):
ZCylinderOut (:3494), ZCylinder (:3305) and Sphere (:4009).

A shape only carries its geometry and voltage; MultiGridB200.installconductor
turns it into per-level ConductorType data through the library's grid-line
intercept code (conductordelfromintercepts, f3d_conductors.F:12).
"""

_condid = [0]


def _next_id():
    _condid[0] += 1
    return _condid[0]


class Conductor:
    kind = None

    def __init__(self, radius, length, voltage, xcent, ycent, zcent, condid=None):
        if not radius > 0:
            raise ValueError("conductor radius must be positive")
        self.radius = float(radius)
        self.length = float(length)
        self.voltage = float(voltage)
        self.xcent, self.ycent, self.zcent = float(xcent), float(ycent), float(zcent)
        self.condid = _next_id() if condid is None else int(condid)


class ZCylinderOut(Conductor):
    """Everything outside radius `radius` of the z axis line through
    (xcent, ycent), for |z - zcent| <= length/2 (a beam pipe)."""
    kind = 0

    def __init__(self, radius, length=1.e30, voltage=0., xcent=0., ycent=0., zcent=0., condid=None):
        super().__init__(radius, length, voltage, xcent, ycent, zcent, condid)


class ZCylinder(Conductor):
    """Solid cylinder along z (e.g. an electrostatic quadrupole rod)."""
    kind = 1

    def __init__(self, radius, length=1.e30, voltage=0., xcent=0., ycent=0., zcent=0., condid=None):
        super().__init__(radius, length, voltage, xcent, ycent, zcent, condid)


class Sphere(Conductor):
    kind = 2

    def __init__(self, radius, voltage=0., xcent=0., ycent=0., zcent=0., condid=None):
        super().__init__(radius, 0., voltage, xcent, ycent, zcent, condid)
