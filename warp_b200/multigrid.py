"""MultiGridB200: the 3D multigrid field solver of scripts/multigrid.py
(MultiGrid3D, :19-955) on one B200, behind the same FieldSolver interface.

A deck switches to it with one line:

    solver = MultiGridB200(nx=..., ..., bounds=[0, 0, 0, 0, 2, 2])   # was MultiGrid3D()
    registersolver(solver)
    solver.installconductor(ZCylinderOut(radius=0.035))

Attributes keep the reference's names and defaults (f3d.v:215-231): mgparam
1.2, mgtol 1e-6 (volts, on max|dphi|), mgmaxiters 100, mgmaxlevels 101,
downpasses = uppasses = 1, lcndbndy True, icndbndy 2; after a solve
mgiters and mgerror hold the last results. Two additions select the B200
forms: precision = "fp64" (the reference's arithmetic) or "mixed" (FP32
V-cycles inside FP64 defect correction), and tolkind = "mgerror" (reference
criterion) or "relres" (max|rhs - A phi| / max|rhs|).

phi and rho are device tensors in the reference layout: phi has shape
(nx+3, ny+3, nz+3) with one guard cell, rho (nx+1, ny+1, nz+1), x fastest
(Fortran order) -- zero-copy views of the solver's own arrays.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .fieldsolver import FieldSolver

_PRECISION = {"fp64": 0, "mixed": 1}
_TOLKIND = {"mgerror": 0, "relres": 1}


def _device_view(ptr, shape, device):
    """Zero-copy float64 tensor over device memory in Fortran order."""
    strides = [8]
    for s in shape[:-1]:
        strides.append(strides[-1] * s)

    class _CAI:
        __cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f8", "data": (int(ptr), False),
                                    "version": 3, "strides": tuple(strides)}

    return torch.as_tensor(_CAI(), device=device)


class MultiGridB200(FieldSolver):
    def __init__(self, nx, ny, nz, xmmin, xmmax, ymmin, ymmax, zmmin, zmmax, bounds=(0, 0, 0, 0, 0, 0),
                 mgparam=1.2, mgtol=1.e-6, mgmaxiters=100, mgmaxlevels=101, downpasses=1, uppasses=1,
                 lcndbndy=True, icndbndy=2, mgform=1, mgverbose=0, precision="fp64", tolkind="mgerror",
                 device=None, use_graphs=True, use_pdl=True, lprecalccoeffs=False):
        if lprecalccoeffs:
            raise NotImplementedError(
                "MultiGridB200: lprecalccoeffs (precalculatecoefficients3d, f3d_mgrid.F:4330) is not supported; "
                "its 9 stored coefficients per node would multiply the HBM traffic of every sweep, so the "
                "coefficients are formed on the fly (the reference's default, lprecalccoeffs = false)")
        if icndbndy != 2:
            raise ValueError("MultiGridB200 supports icndbndy = 2 (quadratic subgrid stencil) only")
        if mgform != 1:
            raise ValueError("mgform: use precision='mixed' for the residual-correction form")
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise ValueError("MultiGridB200 runs on a CUDA device only")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        torch.cuda.set_device(self.device)
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.xmmin, self.xmmax = float(xmmin), float(xmmax)
        self.ymmin, self.ymmax = float(ymmin), float(ymmax)
        self.zmmin, self.zmmax = float(zmmin), float(zmmax)
        self.dx = (self.xmmax - self.xmmin) / self.nx
        self.dy = (self.ymmax - self.ymmin) / self.ny
        self.dz = (self.zmmax - self.zmmin) / self.nz
        self.bounds = list(int(b) for b in bounds)
        self.mgparam, self.mgtol, self.mgmaxiters = float(mgparam), float(mgtol), int(mgmaxiters)
        self.mgmaxlevels, self.downpasses, self.uppasses = int(mgmaxlevels), int(downpasses), int(uppasses)
        self.lcndbndy, self.icndbndy, self.mgform, self.mgverbose = bool(lcndbndy), icndbndy, mgform, mgverbose
        self.precision, self.tolkind = precision, tolkind
        # replay V-cycles from captured CUDA graphs; programmatic dependent
        # launch of the solver's kernels
        self.use_graphs, self.use_pdl = bool(use_graphs), bool(use_pdl)
        self.mgiters, self.mgerror, self.relres, self.converged = 0, 0., -1., True
        self.conductordatalist = []
        self._conductors_installed = False
        self.pgroups = []
        g = _lib.Grid(self.nx, self.ny, self.nz, self.xmmin, self.xmmax, self.ymmin, self.ymmax, self.zmmin,
                      self.zmmax, (ctypes.c_int * 6)(*self.bounds))
        h = ctypes.c_void_p()
        _lib.check(_lib.lib.wg_create(ctypes.byref(g), ctypes.byref(h)))
        self._h = h
        self._bind_stream()
        pphi, prho = ctypes.c_void_p(), ctypes.c_void_p()
        _lib.check(_lib.lib.wg_arrays(h, ctypes.byref(pphi), ctypes.byref(prho)))
        self._phi = _device_view(pphi.value, (self.nx + 3, self.ny + 3, self.nz + 3), self.device)
        self._rho = _device_view(prho.value, (self.nx + 1, self.ny + 1, self.nz + 1), self.device)
        self._lattice = None
        self._lcorrectede = False

    def __del__(self):
        h = getattr(self, "_h", None)
        lib = getattr(_lib, "lib", None)
        if h and lib is not None:
            lib.wg_destroy(h)
            self._h = None

    # -- plumbing -----------------------------------------------------------
    def _bind_stream(self):
        _lib.check(_lib.lib.wg_set_stream(self._h, ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)))

    @property
    def phi(self):
        return self._phi

    @phi.setter
    def phi(self, value):
        self._phi.copy_(torch.as_tensor(value, dtype=torch.float64, device=self.device))

    @property
    def rho(self):
        return self._rho

    @rho.setter
    def rho(self, value):
        self._rho.copy_(torch.as_tensor(value, dtype=torch.float64, device=self.device))

    @property
    def lcorrectede(self):
        """f3d.lcorrectede (f3d.v:152): when True, fetche and advance gather E
        next to conductors from the subgrid data (sete3dwithconductor,
        f3d_mgrid.F:4774-5220) instead of plain centred differences, and
        particles outside the grid get no field. Default False."""
        return self._lcorrectede

    @lcorrectede.setter
    def lcorrectede(self, on):
        _lib.check(_lib.lib.wg_set_correctede(self._h, int(bool(on))))
        self._lcorrectede = bool(on)

    def getphi(self):
        """Host copy of phi on the nodes 0..nx, 0..ny, 0..nz (getphi)."""
        return self._phi[1:-1, 1:-1, 1:-1].cpu().numpy()

    def getrho(self):
        return self._rho.cpu().numpy()

    def levels(self):
        n = ctypes.c_int()
        dims = (ctypes.c_int * 303)()
        d = (ctypes.c_double * 303)()
        _lib.check(_lib.lib.wg_level_info(self._h, ctypes.byref(n), dims, d, 101))
        return [((dims[3 * i], dims[3 * i + 1], dims[3 * i + 2]), (d[3 * i], d[3 * i + 1], d[3 * i + 2]))
                for i in range(n.value)]

    # -- conductors (multigrid.py:743-826) ---------------------------------
    def installconductor(self, conductor, xmin=None, xmax=None, ymin=None, ymax=None, zmin=None, zmax=None,
                         dfill=None):
        """Adds the conductor; its data is generated at the next solve."""
        self.conductordatalist.append((conductor, dfill))
        self._conductors_installed = False

    def uninstallconductor(self, conductor):
        n = len(self.conductordatalist)
        self.conductordatalist = [c for c in self.conductordatalist if c[0] is not conductor]
        if len(self.conductordatalist) == n:
            raise Exception("conductor was not found")
        self._conductors_installed = False

    def setconductorvoltage(self, voltage, condid=0, discrete=False, setvinject=False):
        """setconductorvoltage (multigrid.py:252-260, generateconductors.py:
        2910-3000) for a scalar voltage: every installed conductor with the
        id condid (or the conductor object itself) takes the voltage, and its
        data is regenerated at the next solve. Voltages given per z cell or
        as a function of position, and setvinject (particle injection), are
        not supported here and raise."""
        if setvinject:
            raise NotImplementedError("setconductorvoltage: setvinject (particle injection) is not supported")
        if callable(voltage) or np.ndim(voltage) != 0:
            raise NotImplementedError("setconductorvoltage: only a scalar voltage is supported")
        cid = getattr(condid, "condid", condid)
        hit = False
        for cond, _ in self.conductordatalist:
            if cond.condid == cid:
                cond.voltage = float(voltage)
                hit = True
        if hit:
            self._conductors_installed = False

    def clearconductors(self):
        self.conductordatalist = []
        self._conductors_installed = False

    def hasconductors(self):
        return len(self.conductordatalist) > 0

    def getconductorobject(self):
        """Generates and uploads the conductor data of every MG level
        (getconductorobject, multigrid.py:188-232)."""
        if self._conductors_installed:
            return
        torch.cuda.current_stream(self.device).synchronize()
        _lib.check(_lib.lib.wg_conductors_clear(self._h))
        for cond, dfill in self.conductordatalist:
            _lib.check(_lib.lib.wg_conductors_add_shape(
                self._h, cond.kind, cond.radius, cond.length, cond.voltage, cond.xcent, cond.ycent, cond.zcent,
                cond.condid, 2.0 if dfill is None else float(dfill)))
        _lib.check(_lib.lib.wg_conductors_finalize(self._h))
        self._conductors_installed = True

    def install_conductor_points(self, interior=None, subgrid=None):
        """Installs raw ConductorType data: interior = (indx[n,3], volt[n],
        ilevel[n]); subgrid = (indx[n,3], dels[n,6], volt[n,6], ilevel[n])."""
        self.conductordatalist = []
        _lib.check(_lib.lib.wg_conductors_clear(self._h))
        if interior is not None:
            indx, volt, lev = (np.ascontiguousarray(interior[0], np.int32),
                               np.ascontiguousarray(interior[1], np.float64),
                               np.ascontiguousarray(interior[2], np.int32))
            _lib.check(_lib.lib.wg_conductors_add_points(
                self._h, 0, len(volt), indx.ctypes.data_as(_lib._i32p), None, volt.ctypes.data_as(_lib._dp),
                lev.ctypes.data_as(_lib._i32p)))
        if subgrid is not None:
            indx, dels, volt, lev = (np.ascontiguousarray(subgrid[0], np.int32),
                                     np.ascontiguousarray(subgrid[1], np.float64),
                                     np.ascontiguousarray(subgrid[2], np.float64),
                                     np.ascontiguousarray(subgrid[3], np.int32))
            _lib.check(_lib.lib.wg_conductors_add_points(
                self._h, 1, len(lev), indx.ctypes.data_as(_lib._i32p), dels.ctypes.data_as(_lib._dp),
                volt.ctypes.data_as(_lib._dp), lev.ctypes.data_as(_lib._i32p)))
        _lib.check(_lib.lib.wg_conductors_finalize(self._h))
        self._conductors_installed = True

    def conductor_data(self):
        """Host copy of the finalized conductor lists (for inspection)."""
        c = np.zeros(3, np.int64)
        _lib.check(_lib.lib.wg_conductors_counts(self._h, c.ctypes.data_as(_lib._i64p)))
        out = {}
        n = int(c[0])
        indx, volt, lev = np.zeros((n, 3), np.int32), np.zeros(n), np.zeros(n, np.int32)
        _lib.check(_lib.lib.wg_conductors_export(self._h, 0, indx.ctypes.data_as(_lib._i32p), None,
                                                 volt.ctypes.data_as(_lib._dp), lev.ctypes.data_as(_lib._i32p)))
        out["interior"] = (indx, volt, lev)
        parts = []
        for which in (1, 2):
            n = int(c[which])
            p = (np.zeros((n, 3), np.int32), np.zeros((n, 6)), np.zeros((n, 6)), np.zeros(n, np.int32))
            _lib.check(_lib.lib.wg_conductors_export(self._h, which, p[0].ctypes.data_as(_lib._i32p),
                                                     p[1].ctypes.data_as(_lib._dp), p[2].ctypes.data_as(_lib._dp),
                                                     p[3].ctypes.data_as(_lib._i32p)))
            parts.append(p)
        out["subgrid"] = tuple(np.concatenate([p[k] for p in parts]) for k in range(4))
        return out

    # -- source, solve, field ----------------------------------------------
    def addpgroup(self, pgroup):
        if pgroup not in self.pgroups:
            self.pgroups.append(pgroup)

    def loadrho(self, pgroups=None, lzero=True, lfinalize_rho=True):
        """loadrho -> setsourcep -> setrho3d (fieldsolver.py:1333,
        multigrid.py:472-511, w3d.F:7757): fixed-point CIC deposit of every
        group, then applyrhoboundaryconditions3d."""
        self._bind_stream()
        groups = self.pgroups if pgroups is None else pgroups
        first = bool(lzero)
        if not groups and lzero:
            self._rho.zero_()
        for pg in groups:
            s = pg.cstruct()
            _lib.check(pg.fn("wg_deposit")(self._h, ctypes.byref(s), int(first)))
            first = False
        if lfinalize_rho:
            _lib.check(_lib.lib.wg_finalize_rho(self._h))

    def deposit_begin(self):
        """Opens a deposit in pieces (wg_deposit_begin): clears the
        fixed-point accumulator. No host synchronization."""
        self._bind_stream()
        _lib.check(_lib.lib.wg_deposit_begin(self._h))

    def deposit_add(self, pgroup, start=0, stop=None):
        """Accumulates particles start:stop of pgroup (wg_deposit_add)."""
        self._bind_stream()
        s = pgroup.cstruct(start, stop)
        _lib.check(pgroup.fn("wg_deposit_add")(self._h, ctypes.byref(s)))

    def deposit_end(self, zero_first=True, lfinalize_rho=True):
        """Converts the accumulated pieces into rho (replacing it when
        zero_first) and applies the rho boundary conditions. The result is
        the same as loadrho of all pieces at once, bit for bit; an
        accumulator overflow is reported by the next solve."""
        self._bind_stream()
        _lib.check(_lib.lib.wg_deposit_end(self._h, int(bool(zero_first))))
        if lfinalize_rho:
            _lib.check(_lib.lib.wg_finalize_rho(self._h))

    def _opts(self):
        flags = (_lib.SOLVE_GRAPH if self.use_graphs else 0) | (_lib.SOLVE_PDL if self.use_pdl else 0)
        return _lib.SolveOpts(self.mgparam, self.mgtol, self.mgmaxiters, self.mgmaxlevels, self.downpasses,
                              self.uppasses, int(self.lcndbndy), _PRECISION[self.precision],
                              _TOLKIND[self.tolkind], flags, int(getattr(self, "mgmaxvcycles", 0)))

    def solve(self, iwhich=0):
        """dosolve -> multigrid3dsolve (multigrid.py:846-917,
        f3d_mgrid.F:83-500). phi is the warm start and the result."""
        if iwhich > 0:
            return
        self._bind_stream()
        self.getconductorobject()
        st = _lib.SolveStats()
        o = self._opts()
        _lib.check(_lib.lib.wg_solve(self._h, ctypes.byref(o), ctypes.byref(st)))
        self.mgiters, self.mgerror, self.relres, self.converged = st.mgiters, st.mgerror, st.relres, bool(st.converged)
        if self.mgverbose >= 1 or (self.mgverbose >= 0 and not self.converged):
            if not self.converged:
                print("Multigrid: Maximum number of iterations reached")
            print("Multigrid: Error converged to %11.3e in %5d v-cycles" %
                  (self.mgerror if self.tolkind == "mgerror" else self.relres, self.mgiters))

    dosolve = solve

    def find_mgparam(self, lsavephi=False, resetpasses=1, log=print):
        """MultiGrid3D.find_mgparam (multigrid.py:827-831,
        find_mgparam.py:28-237): tunes mgparam, downpasses and uppasses for
        the fastest solve of the problem the solver holds."""
        from .find_mgparam import find_mgparam
        return find_mgparam(self, lsavephi=lsavephi, resetpasses=resetpasses, log=log)

    def relresidual(self):
        self._bind_stream()
        self.getconductorobject()
        out = ctypes.c_double()
        _lib.check(_lib.lib.wg_relresidual(self._h, self.mgparam, ctypes.byref(out)))
        return out.value

    def getese(self):
        """Electrostatic energy dx dy dz / 2 * sum(rho * phi) over the nodes
        (MultiGrid3D.getese -> getese3dfromrhophi, multigrid.py:447-469,
        dw3d.F:708-777). Returns a float (the reference stores it in top.ese)."""
        self._bind_stream()
        out = ctypes.c_double()
        _lib.check(_lib.lib.wg_field_energy(self._h, ctypes.byref(out)))
        return out.value

    def residual_field(self, out=None):
        """rhs - A phi of the current phi (conductor voltages imposed), in the
        rho layout: the right-hand side of the residual-correction equation,
        in volts per SOR update. Returns a float64 device tensor indexed
        [ix, iy, iz]."""
        self._bind_stream()
        self.getconductorobject()
        n = (self.nx + 1) * (self.ny + 1) * (self.nz + 1)
        if out is None:
            out = torch.empty(n, dtype=torch.float64, device=self.device)
        _lib.check(_lib.lib.wg_residual_field(self._h, self.mgparam, ctypes.c_void_p(out.data_ptr())))
        return out.view(self.nz + 1, self.ny + 1, self.nx + 1).permute(2, 1, 0)

    def fetche(self, pgroup=None, ipmin=None, np=None):
        """fetche -> fetchfieldfrompositions -> sete3d (multigrid.py:521-558,
        w3d.F:3963): E at the particles, written to pgroup.ex/ey/ez.

        ipmin (1-based) and np select the particles ipmin .. ipmin+np-1 of
        one group, the slice that WARP's fetche3d zeroes and hands to the
        registered solver (w3d.ipminfsapi, w3d.npfsapi; fieldsolver.py:
        1434-1511, w3d.F:10978-11060); E outside the slice is left as it is."""
        self._bind_stream()
        if self._lcorrectede:
            self.getconductorobject()
        if ipmin is not None or np is not None:
            if pgroup is None or ipmin is None or np is None:
                raise ValueError("fetche: a particle slice needs pgroup, ipmin and np")
            i0, n = int(ipmin) - 1, int(np)
            if i0 < 0 or n < 0 or i0 + n > pgroup.np:
                raise ValueError("fetche: slice %d..%d outside the %d particles" % (i0 + 1, i0 + n, pgroup.np))
            views = [getattr(pgroup, k)[i0:i0 + n] for k in ("x", "y", "z", "ex", "ey", "ez")]
        else:
            groups = self.pgroups if pgroup is None else [pgroup]
            views = None
        for v in ([views] if views is not None else
                  [[getattr(pg, k) for k in ("x", "y", "z", "ex", "ey", "ez")] for pg in groups]):
            n = int(v[0].shape[0])
            # the gather reads FP64 positions (FP32 groups are widened)
            v = [t.double().contiguous() for t in v[:3]] + v[3:]
            for e in v[3:]:
                e.zero_()
            if n:
                _lib.check(_lib.lib.wg_fetch_e(self._h, *(t.data_ptr() for t in v), n))

    fetchfieldfrompositions = fetche

    def fetche_host(self, x, y, z):
        """E at host positions (numpy arrays), returned as three host arrays:
        the call a host-array caller such as WARP's own
        fetchfieldfrompositions (multigrid.py:521-558) makes. Positions are
        copied in, the gather runs on the device, the fields are copied out."""
        self._bind_stream()
        if self._lcorrectede:
            self.getconductorobject()
        pos = [torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(self.device) for a in (x, y, z)]
        n = int(pos[0].shape[0])
        e = torch.zeros((3, n), dtype=torch.float64, device=self.device)
        if n:
            _lib.check(_lib.lib.wg_fetch_e(self._h, pos[0].data_ptr(), pos[1].data_ptr(), pos[2].data_ptr(),
                                           e[0].data_ptr(), e[1].data_ptr(), e[2].data_ptr(), n))
        return e.cpu().numpy()

    # -- drop-in particle advance ------------------------------------------
    def setlattice(self, lattice, nzl=None, zlmin=None, dzl=None):
        """Installs the quad tables of `lattice` (warp_b200.lattice.Lattice)
        on lattice cells of size dzl (default dz) covering the grid."""
        dzl = self.dz if dzl is None else float(dzl)
        zlmin = self.zmmin if zlmin is None else float(zlmin)
        nzl = int(round((self.zmmax - zlmin) / dzl)) + 1 if nzl is None else int(nzl)
        czs, cze, cdb = (np.ascontiguousarray(a) for a in lattice.tables(zlmin, dzl, nzl))
        _lib.check(_lib.lib.wg_set_lattice(self._h, czs.ctypes.data_as(_lib._dp), cze.ctypes.data_as(_lib._dp),
                                           cdb.ctypes.data_as(_lib._dp), nzl, zlmin, dzl))
        self._lattice = (czs, cze, cdb, nzl, zlmin, dzl)

    def advance(self, pgroup, dt, prwall=1.e30, prwallx=0., prwally=0., start=0, stop=None, center="fullv",
                deposit=False):
        """One fused particle advance of padvnc3d (w3d.F:1575) plus
        particleboundaries3d: gather E from phi, quad B (if a lattice is
        installed), the velocity push and drift that center selects, the
        periodic z wrap and the round absorbing pipe of radius prwall.
        center "fullv" (w3d.F:1862-1987): half E kick, Boris rotation, half
        E kick, drift. "halfv" (w3d.F:1989-2125), the first step after
        loading, when velocities are still at the positions' time: half-dt
        rotation, half E kick, drift. "synchv" (w3d.F:2187-2310): half E kick
        and half-dt rotation only, bringing velocities back to the
        positions' time. start/stop restrict it to a range of the group's
        particles. With deposit=True the advanced particles' charge is also
        added to the deposit opened by deposit_begin(), in the same pass
        (wg_advance_deposit): rho after deposit_end() is the same, bit for
        bit, as a loadrho() of the advanced particles."""
        if center not in _lib.CENTERS:
            raise ValueError("center must be one of %s" % sorted(_lib.CENTERS))
        self._bind_stream()
        if self._lcorrectede:
            self.getconductorobject()
        s = pgroup.cstruct(start, stop)
        p = _lib.PushParams(float(dt), float(prwall), float(prwallx), float(prwally),
                            int(self._lattice is not None), _lib.CENTERS[center])
        _lib.check(pgroup.fn("wg_advance_deposit" if deposit else "wg_advance")(self._h, ctypes.byref(s),
                                                                                ctypes.byref(p)))

    def zmoments(self, pgroup, uold, dt, zmmntmin, zmmntmax, nzmmnt, zbeam=0., dtscale=1., zmmntdtextmax=1e36):
        """The moment sums of getzmmnt (wg_zmoments): returns zmmnts0 (33,)
        over all live particles and zmmnts (nzmmnt+1, 33) on the z grid.
        uold is a triple of device arrays with the velocities dt earlier (the
        reference takes them before the synchv half step, with dt = dt/2).
        warp_b200.diagnostics.finalize turns the sums into moments."""
        self._bind_stream()
        s = pgroup.cstruct()
        z0 = np.zeros(33)
        zm = np.zeros((int(nzmmnt) + 1, 33))
        dp = ctypes.POINTER(ctypes.c_double)
        uold = [u.to(pgroup.dtype).contiguous() for u in uold]  # kept alive across the call
        uo = [ctypes.c_void_p(u.data_ptr()) for u in uold]
        _lib.check(pgroup.fn("wg_zmoments")(self._h, ctypes.byref(s), uo[0], uo[1], uo[2], float(dt), float(dtscale),
                                        float(zbeam), float(zmmntmin), float(zmmntmax), int(nzmmnt),
                                        float(zmmntdtextmax), z0.ctypes.data_as(dp), zm.ctypes.data_as(dp)))
        return z0, zm

    def moments(self, pgroup):
        """Global moments of live particles: dict n, xbar, ybar, xrms, yrms,
        epsx, epsy (getzmmnt, top.F:521-1444)."""
        self._bind_stream()
        s = pgroup.cstruct()
        out = (ctypes.c_double * 8)()
        _lib.check(pgroup.fn("wg_moments")(self._h, ctypes.byref(s), out))
        keys = ("n", "xbar", "ybar", "xrms", "yrms", "epsx", "epsy")
        return {k: out[i] for i, k in enumerate(keys)}


MultiGrid3D = MultiGridB200


class FullMultiGridB200(MultiGridB200):
    """FullMultiGrid3D (scripts/multigrid.py:957-1020): each solve is a full
    multigrid (fullmultigrid3dsolve, f3d_mgrid.F:502-945). The source is
    restricted to every level, the coarsest level is solved first, and each
    finer level starts from the expanded coarse phi and does mgmaxvcycles
    V-cycles (default 2); the finest level then iterates to mgtol as
    MultiGrid3D does. The previous phi is not used as a starting point."""

    def __init__(self, *args, mgmaxvcycles=2, **kw):
        if int(mgmaxvcycles) < 1:
            raise ValueError("mgmaxvcycles must be at least 1")
        self.mgmaxvcycles = int(mgmaxvcycles)
        super().__init__(*args, **kw)


FullMultiGrid3D = FullMultiGridB200
