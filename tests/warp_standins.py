"""Stand-ins for the WARP objects the binding meets (warp_b200/warp_binding.py),
with the reference's names, signatures and attribute handling: the conductor
classes of scripts/generateconductors.py (Assembly's condid='next' counter,
ZCylinderOut's zlower/zupper, :236-280, :3305, :3494, :4009), the host arrays
and conductor list of scripts/multigrid.py's MultiGrid3D (:77-330, 743-751),
and the top/f3d package globals it reads. WARP itself (Python 2 + Forthon)
does not run here; these carry only what the binding touches."""
import numpy as np


class Assembly:
    nextcondid = 1

    def __init__(self, v=0., x=0., y=0., z=0., condid="next"):
        self.voltage = v
        self.xcent, self.ycent, self.zcent = x, y, z
        if condid == "next":
            self.condid = Assembly.nextcondid
            Assembly.nextcondid += 1
        else:
            self.condid = condid


class ZCylinderOut(Assembly):
    def __init__(self, radius, length=None, voltage=0., xcent=0., ycent=0., zcent=0., condid="next", zlower=None,
                 zupper=None):
        if zlower is not None and zupper is not None:
            length = zupper - zlower
            zcent = 0.5 * (zlower + zupper)
            self.zlower, self.zupper = zlower, zupper
        assert length is not None
        Assembly.__init__(self, voltage, xcent, ycent, zcent, condid)
        self.radius, self.length = radius, length


class ZCylinder(ZCylinderOut):
    pass


class Sphere(Assembly):
    def __init__(self, radius, voltage=0., xcent=0., ycent=0., zcent=0., condid="next"):
        Assembly.__init__(self, voltage, xcent, ycent, zcent, condid)
        self.radius = radius


class Box(Assembly):
    def __init__(self, xsize, ysize, zsize, voltage=0., xcent=0., ycent=0., zcent=0., condid="next"):
        Assembly.__init__(self, voltage, xcent, ycent, zcent, condid)
        self.xsize, self.ysize, self.zsize = xsize, ysize, zsize


class top:
    efetch = np.array([1])
    wpid = 0


class w3d:
    pass


class f3d:
    lcorrectede = False


class MultiGrid3D:
    """What the binding uses of scripts/multigrid.py's MultiGrid3D: the mesh
    and solver attributes, the host source and guarded potential arrays, and
    the conductor list."""

    def __init__(self, nx=32, ny=32, nz=48, xmmin=-0.5, xmmax=0.5, ymmin=-0.5, ymmax=0.5, zmmin=-0.5, zmmax=0.5,
                 bounds=(0, 0, 0, 0, 2, 2), mgparam=1.2, mgtol=1e-6, mgmaxiters=100, mgmaxlevels=101,
                 downpasses=1, uppasses=1, lcndbndy=1):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.xmmin, self.xmmax, self.ymmin, self.ymmax, self.zmmin, self.zmmax = (xmmin, xmmax, ymmin, ymmax,
                                                                                  zmmin, zmmax)
        self.dx, self.dy, self.dz = (xmmax - xmmin) / nx, (ymmax - ymmin) / ny, (zmmax - zmmin) / nz
        self.bounds = np.array(bounds)
        self.mgparam, self.mgtol, self.mgmaxiters, self.mgmaxlevels = mgparam, mgtol, mgmaxiters, mgmaxlevels
        self.downpasses, self.uppasses, self.lcndbndy = downpasses, uppasses, lcndbndy
        self.nxguardphi, self.nxguardrho, self.mgform = 1, 0, 1
        self.source = np.zeros((nx + 1, ny + 1, nz + 1), order="F")
        self.sourcep = self.source
        self.potential = np.zeros((nx + 3, ny + 3, nz + 3), order="F")
        self.conductordatalist = []
        self.mgiters, self.mgerror = 0, 0.

    def installconductor(self, conductor, xmin=None, xmax=None, ymin=None, ymax=None, zmin=None, zmax=None,
                         dfill=None):
        self.conductordatalist.append((conductor, xmin, xmax, ymin, ymax, zmin, zmax, dfill))

    def uninstallconductor(self, conductor):
        n = len(self.conductordatalist)
        self.conductordatalist = [c for c in self.conductordatalist if c[0] is not conductor]
        if len(self.conductordatalist) == n:
            raise Exception("conductor was not found")

    def getphi(self):
        return self.potential[1:-1, 1:-1, 1:-1]
