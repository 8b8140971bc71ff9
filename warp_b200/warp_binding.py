"""The WARP-side binding: a subclass of WARP's own MultiGrid3D
(scripts/multigrid.py:19-955) whose deposit, field solve and gather run in
libwarp_b200, for WARP's solver objects, host arrays and conductor classes.

A WARP deck switches with one line:

    from warp import *
    from warp.field_solvers import multigrid
    from warp_b200.warp_binding import gpu_multigrid
    MultiGrid3D = gpu_multigrid(multigrid.MultiGrid3D, top, w3d, f3d)  # the added line
    solver = MultiGrid3D()
    registersolver(solver)                                            # scripts/fieldsolver.py:173
    solver.installconductor(ZCylinderOut(radius=0.035, zlower=0., zupper=1.))

WARP keeps calling the methods it always calls:
- setsourcepatposition (multigrid.py:492-519, setrho3d) from its loadrho:
  each batch of particles is deposited on the GPU (64-bit fixed point) and
  added to WARP's host source array, so WARP's own finalize (rho boundary
  conditions, sourcep -> source) works unchanged;
- dosolve (multigrid.py:846-917, multigrid3dsolve): WARP's source and its
  guarded potential (the warm start) go to the device, the solve runs there,
  and the whole guarded potential, guard cells included, comes back;
- fetchfieldfrompositions (multigrid.py:521-558, sete3d or
  sete3dwithconductor with efetch = 1): E at host positions from the device
  phi, added to WARP's ex, ey, ez as sete3d does;
- installconductor (multigrid.py:743-751): WARP's conductor objects are kept
  in WARP's list and translated, by class, into the library's shapes
  (shape_from_warp).

What it does not cover raises NotImplementedError: conductor classes other
than ZCylinderOut, ZCylinder and Sphere, installing into a sub-box,
per-particle weights (setrho3dw, top.wpid != 0), a moving grid (zgrid != 0),
efetch other than 1, guard-cell counts other than nxguardphi = 1 and
nxguardrho = 0, and mgform 2 (use precision="mixed" for the residual
correction form).
"""
import numpy as np

from . import conductors as _shapes

_CLASSES = {"ZCylinderOut": _shapes.ZCylinderOut, "ZCylinder": _shapes.ZCylinder, "Sphere": _shapes.Sphere}


def shape_from_warp(conductor):
    """The warp_b200 shape for a WARP conductor object. The class is
    recognised by name and the geometry read from the attributes
    generateconductors.py sets (radius, length or zlower/zupper, voltage,
    xcent, ycent, zcent, condid; :3305 ZCylinder, :3494 ZCylinderOut, :4009
    Sphere). The condid is WARP's, which has already resolved 'next'."""
    name = type(conductor).__name__
    if name not in _CLASSES:
        raise NotImplementedError("warp_b200: conductor class %s is not supported (ZCylinderOut, ZCylinder and "
                                  "Sphere are)" % name)
    condid = getattr(conductor, "condid", None)
    if not isinstance(condid, (int, np.integer)):
        raise ValueError("warp_b200: conductor %s has no integer condid" % name)
    common = dict(voltage=float(conductor.voltage), xcent=float(conductor.xcent), ycent=float(conductor.ycent),
                  condid=int(condid))
    if name == "Sphere":
        return _shapes.Sphere(radius=float(conductor.radius), zcent=float(conductor.zcent), **common)
    zlower, zupper = getattr(conductor, "zlower", None), getattr(conductor, "zupper", None)
    if zlower is not None and zupper is not None:
        length, zcent = float(zupper) - float(zlower), 0.5 * (float(zlower) + float(zupper))
    else:
        if getattr(conductor, "length", None) is None:
            raise ValueError("warp_b200: %s needs a length or both zlower and zupper" % name)
        length, zcent = float(conductor.length), float(conductor.zcent)
    return _CLASSES[name](radius=float(conductor.radius), length=length, zcent=zcent, **common)


def gpu_multigrid(RefMG, top, w3d, f3d, **gpu_options):
    """A subclass of WARP's MultiGrid3D class RefMG whose setsourcepatposition,
    dosolve and fetchfieldfrompositions run on the GPU. top, w3d and f3d are
    WARP's Forthon packages (the module globals multigrid.py reads).
    gpu_options go to MultiGridB200 (precision, tolkind, device, ...)."""
    from .multigrid import MultiGridB200

    class MultiGrid3D(RefMG):
        __doc__ = "MultiGrid3D with its deposit, solve and gather in libwarp_b200.\n\n" + (RefMG.__doc__ or "")

        def __init__(self, *args, **kw):
            RefMG.__init__(self, *args, **kw)
            if getattr(self, "nxguardphi", 1) != 1 or getattr(self, "nxguardrho", 0) != 0:
                raise NotImplementedError("warp_b200: needs nxguardphi = 1 and nxguardrho = 0")
            if getattr(self, "mgform", 1) != 1:
                raise NotImplementedError("warp_b200: mgform 2; use precision='mixed' for residual correction")
            self._gpu = MultiGridB200(self.nx, self.ny, self.nz, self.xmmin, self.xmmax, self.ymmin, self.ymmax,
                                      self.zmmin, self.zmmax, bounds=tuple(int(b) for b in self.bounds),
                                      mgparam=self.mgparam, mgtol=self.mgtol, mgmaxiters=self.mgmaxiters,
                                      mgmaxlevels=self.mgmaxlevels, downpasses=self.downpasses,
                                      uppasses=self.uppasses, lcndbndy=bool(self.lcndbndy), mgverbose=-1,
                                      **gpu_options)

        def installconductor(self, conductor, xmin=None, xmax=None, ymin=None, ymax=None, zmin=None, zmax=None,
                             dfill=None):
            if any(v is not None for v in (xmin, xmax, ymin, ymax, zmin, zmax)):
                raise NotImplementedError("warp_b200: installing a conductor into a sub-box")
            shape = shape_from_warp(conductor)
            RefMG.installconductor(self, conductor, xmin=xmin, xmax=xmax, ymin=ymin, ymax=ymax, zmin=zmin,
                                   zmax=zmax, dfill=dfill)
            self._gpu.installconductor(shape, dfill=dfill)

        def uninstallconductor(self, conductor):
            RefMG.uninstallconductor(self, conductor)
            self._gpu.conductordatalist = [(shape_from_warp(c[0]), c[-1]) for c in self.conductordatalist]
            self._gpu._conductors_installed = False

        def setsourcepatposition(self, x, y, z, ux, uy, uz, gaminv, wfact, zgrid, q, w, depos_order):
            n = len(x)
            if n == 0:
                return
            if getattr(top, "wpid", 0) != 0:
                raise NotImplementedError("warp_b200: per-particle weights (setrho3dw)")
            if zgrid != 0.:
                raise NotImplementedError("warp_b200: a moving grid (zgrid != 0)")
            import torch
            from .particles import ParticleGroup
            g = np.ones(n) if gaminv is None or len(gaminv) != n else gaminv
            pg = ParticleGroup({"x": x, "y": y, "z": z, "ux": ux, "uy": uy, "uz": uz, "gaminv": g}, q=q, w=w,
                               device=self._gpu.device, with_fields=False)
            # this batch alone on the device, then added to WARP's host source
            self._gpu.loadrho(pgroups=[pg], lzero=True, lfinalize_rho=False)
            torch.cuda.current_stream(self._gpu.device).synchronize()
            self.sourcep[...] += self._gpu.rho.cpu().numpy()

        def dosolve(self, iwhich=0, *args):
            if iwhich > 0:
                return
            if getattr(self, "l_internal_dosolve", True) is False:
                return
            if self.potential.shape != (self.nx + 3, self.ny + 3, self.nz + 3):
                raise NotImplementedError("warp_b200: potential of shape %s" % (self.potential.shape,))
            self._gpu.mgparam, self._gpu.mgtol, self._gpu.mgmaxiters = self.mgparam, self.mgtol, self.mgmaxiters
            self._gpu.downpasses, self._gpu.uppasses = self.downpasses, self.uppasses
            self._gpu.rho = self.source
            self._gpu.phi = self.potential           # WARP's potential is the warm start
            self._gpu.solve()
            self.potential[...] = self._gpu.phi.cpu().numpy()
            self.mgiters, self.mgerror = self._gpu.mgiters, self._gpu.mgerror

        def fetchfieldfrompositions(self, x, y, z, ex, ey, ez, bx, by, bz, js=0, pgroup=None):
            n = len(x)
            if n == 0:
                return
            if int(top.efetch[js]) != 1:
                raise NotImplementedError("warp_b200: efetch = %d (only 1 is built)" % int(top.efetch[js]))
            self._gpu.lcorrectede = bool(getattr(f3d, "lcorrectede", False))
            e = self._gpu.fetche_host(x, y, z)
            ex += e[0]
            ey += e[1]
            ez += e[2]

    return MultiGrid3D
