"""ctypes wrapper of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker. The warp_b200 package never
imports it.

All grids are numpy arrays in the reference's Fortran layout (x fastest):
phi has shape (nx+3, ny+3, nz+3) (one guard cell), rho (nx+1, ny+1, nz+1).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_i64p = ctypes.POINTER(ctypes.c_int64)


def build():
    """Compiles liboracle.so with make (gcc is all it needs)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        src = os.path.join(_HERE, "oracle.cpp")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(path)
        L.or_mglevels.restype = ctypes.c_int
        L.or_mglevels.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [_ip, _dp, ctypes.c_int]
        L.or_cond_new.restype = ctypes.c_void_p
        L.or_cond_new.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3
        L.or_cond_free.argtypes = [ctypes.c_void_p]
        L.or_cond_add_shape.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.c_double] * 6 + \
            [ctypes.c_int] + [ctypes.c_double] * 4
        L.or_cond_add_points.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, _ip, _dp, _dp, _ip]
        L.or_cond_finalize.argtypes = [ctypes.c_void_p]
        L.or_cond_counts.argtypes = [ctypes.c_void_p, _i64p]
        L.or_cond_export.argtypes = [ctypes.c_void_p, ctypes.c_int, _ip, _dp, _dp, _ip]
        L.or_mgsolve.restype = ctypes.c_int
        L.or_mgsolve.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [_ip, _dp, _dp, ctypes.c_void_p,
                                 ctypes.c_double, ctypes.c_double] + [ctypes.c_int] * 6 + [_ip, _dp, ctypes.c_int]
        L.or_relresidual.restype = ctypes.c_double
        L.or_relresidual.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [_ip, _dp, _dp, ctypes.c_void_p,
                                     ctypes.c_double]
        L.or_setrho.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 7 + [_dp, ctypes.c_int64, _dp, _dp, _dp,
                                _dp, ctypes.c_double, ctypes.c_double]
        L.or_rhobc.argtypes = [ctypes.c_int] * 3 + [_dp, _ip]
        L.or_sete.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 7 + [_dp, ctypes.c_int64] + [_dp] * 6
        L.or_quad_table.argtypes = [ctypes.c_int, _dp, _dp, _dp] + [ctypes.c_double] * 4 + [ctypes.c_int] + [_dp] * 3
        L.or_push.argtypes = [ctypes.c_int, ctypes.c_int64] + [_dp] * 10 + [ctypes.c_double] * 3 + [_dp] * 3 + \
            [ctypes.c_int] + [ctypes.c_double] * 7
        L.or_moments.argtypes = [ctypes.c_int64] + [_dp] * 6 + [_dp]
        L.or_zmoments.argtypes = [ctypes.c_int64] + [_dp] * 10 + [ctypes.c_double] * 5 + [ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.or_sete_cond.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 3 + [ctypes.c_double] * 7 + \
            [_dp, ctypes.c_int64] + [_dp] * 6
        L.or_eps0.restype = ctypes.c_double
        L.or_threads.restype = ctypes.c_int
        L.or_ese.argtypes = [ctypes.c_int] * 3 + [_dp, _dp] + [ctypes.c_double] * 3
        L.or_ese.restype = ctypes.c_double
        _LIB = L
    return _LIB


def _d(a):
    assert a.dtype == np.float64 and (a.flags.f_contiguous or a.ndim == 1 or a.flags.c_contiguous)
    return a.ctypes.data_as(_dp)


def _i(a):
    assert a.dtype == np.int32
    return a.ctypes.data_as(_ip)


def eps0():
    return lib().or_eps0()


def mglevels(nx, ny, nz, dx, dy, dz):
    n = np.zeros(3 * 101, np.int32)
    d = np.zeros(3 * 101, np.float64)
    k = lib().or_mglevels(nx, ny, nz, dx, dy, dz, _i(n), _d(d), 101)
    return [(tuple(int(v) for v in n[3 * i:3 * i + 3]), tuple(float(v) for v in d[3 * i:3 * i + 3]))
            for i in range(k)]


class Conductors:
    """Conductor data of the oracle (ConductorType layout, f3d.v:105-164)."""

    SHAPES = {"ZCylinderOut": 0, "ZCylinder": 1, "Sphere": 2}

    def __init__(self, nx, ny, nz, dx, dy, dz, xmmin, ymmin, zmmin):
        self.h = lib().or_cond_new(nx, ny, nz, dx, dy, dz)
        self.mins = (xmmin, ymmin, zmmin)
        self.finalized = False

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_cond_free(self.h)
            self.h = None

    def add_shape(self, kind, radius, length=0.0, voltage=0.0, xcent=0.0, ycent=0.0, zcent=0.0, condid=1,
                  dfill=2.0):
        lib().or_cond_add_shape(self.h, self.SHAPES[kind], radius, length, voltage, xcent, ycent, zcent, condid,
                                self.mins[0], self.mins[1], self.mins[2], dfill)

    def add_points(self, interior=None, subgrid=None):
        if interior is not None:
            indx, volt, ilevel = interior
            indx = np.ascontiguousarray(indx, np.int32)
            volt = np.ascontiguousarray(volt, np.float64)
            ilevel = np.ascontiguousarray(ilevel, np.int32)
            lib().or_cond_add_points(self.h, 0, len(volt), _i(indx), None, _d(volt), _i(ilevel))
        if subgrid is not None:
            indx, dels, volt, ilevel = subgrid
            indx = np.ascontiguousarray(indx, np.int32)
            dels = np.ascontiguousarray(dels, np.float64)
            volt = np.ascontiguousarray(volt, np.float64)
            ilevel = np.ascontiguousarray(ilevel, np.int32)
            lib().or_cond_add_points(self.h, 1, len(ilevel), _i(indx), _d(dels), _d(volt), _i(ilevel))

    def finalize(self):
        lib().or_cond_finalize(self.h)
        self.finalized = True

    def export(self):
        """Returns dict with interior (indx[n,3], volt[n], ilevel[n]) and
        subgrid (indx[n,3], dels[n,6], volt[n,6], ilevel[n]) for even+odd."""
        c = np.zeros(3, np.int64)
        lib().or_cond_counts(self.h, c.ctypes.data_as(_i64p))
        out = {}
        n = int(c[0])
        indx = np.zeros((n, 3), np.int32)
        volt = np.zeros(n, np.float64)
        lev = np.zeros(n, np.int32)
        if n:
            lib().or_cond_export(self.h, 0, _i(indx), None, _d(volt), _i(lev))
        out["interior"] = (indx, volt, lev)
        parts = []
        for which in (1, 2):
            n = int(c[which])
            indx = np.zeros((n, 3), np.int32)
            dels = np.zeros((n, 6), np.float64)
            volt = np.zeros((n, 6), np.float64)
            lev = np.zeros(n, np.int32)
            if n:
                lib().or_cond_export(self.h, which, _i(indx), _d(dels), _d(volt), _i(lev))
            parts.append((indx, dels, volt, lev))
        out["subgrid"] = tuple(np.concatenate([p[k] for p in parts]) for k in range(4))
        return out


def mgsolve(phi, rho, dx, dy, dz, bounds, conductors=None, mgparam=1.2, mgtol=1e-6, mgmaxiters=100,
            mgmaxlevels=101, downpasses=1, uppasses=1, mgform=1, lcndbndy=True, mgmaxvcycles=0):
    """multigrid3dsolve on the CPU; phi updated in place. Returns (iters, err).
    mgmaxvcycles > 0 selects fullmultigrid3dsolve with that many V-cycles
    per coarse level (FullMultiGrid3D's default is 2)."""
    nx, ny, nz = rho.shape[0] - 1, rho.shape[1] - 1, rho.shape[2] - 1
    assert phi.shape == (nx + 3, ny + 3, nz + 3) and phi.flags.f_contiguous and rho.flags.f_contiguous
    b = np.ascontiguousarray(bounds, np.int32)
    it = ctypes.c_int(0)
    err = ctypes.c_double(0.0)
    rc = lib().or_mgsolve(nx, ny, nz, dx, dy, dz, _i(b), _d(phi), _d(rho),
                          conductors.h if conductors is not None else None, mgparam, mgtol, mgmaxiters,
                          mgmaxlevels, downpasses, uppasses, mgform, int(lcndbndy), ctypes.byref(it),
                          ctypes.byref(err), int(mgmaxvcycles))
    if rc != 0:
        raise RuntimeError("oracle mgsolve failed: %d" % rc)
    return it.value, err.value


def relresidual(phi, rho, dx, dy, dz, bounds, conductors=None, mgparam=1.2):
    nx, ny, nz = rho.shape[0] - 1, rho.shape[1] - 1, rho.shape[2] - 1
    b = np.ascontiguousarray(bounds, np.int32)
    return lib().or_relresidual(nx, ny, nz, dx, dy, dz, _i(b), _d(phi), _d(rho),
                                conductors.h if conductors is not None else None, mgparam)


def setrho(rho, x, y, z, q, w, dx, dy, dz, xmmin, ymmin, zmmin, gaminv=None, zgrid=0.0):
    nx, ny, nz = rho.shape[0] - 1, rho.shape[1] - 1, rho.shape[2] - 1
    lib().or_setrho(nx, ny, nz, dx, dy, dz, xmmin, ymmin, zmmin, zgrid, _d(rho), len(x), _d(x), _d(y), _d(z),
                    _d(gaminv) if gaminv is not None else None, q, w)


def rhobc(rho, bounds):
    nx, ny, nz = rho.shape[0] - 1, rho.shape[1] - 1, rho.shape[2] - 1
    b = np.ascontiguousarray(bounds, np.int32)
    lib().or_rhobc(nx, ny, nz, _d(rho), _i(b))


def sete(phi, x, y, z, dx, dy, dz, xmmin, ymmin, zmmin, zgrid=0.0):
    nx, ny, nz = phi.shape[0] - 3, phi.shape[1] - 3, phi.shape[2] - 3
    n = len(x)
    ex = np.zeros(n)
    ey = np.zeros(n)
    ez = np.zeros(n)
    lib().or_sete(nx, ny, nz, dx, dy, dz, xmmin, ymmin, zmmin, zgrid, _d(phi), n, _d(x), _d(y), _d(z), _d(ex),
                  _d(ey), _d(ez))
    return ex, ey, ez


def quad_tables(zs, ze, db, zlatperi, zlatstrt, zlmin, dzl, nzl):
    zs = np.ascontiguousarray(zs, np.float64)
    ze = np.ascontiguousarray(ze, np.float64)
    db = np.ascontiguousarray(db, np.float64)
    czs = np.zeros(nzl + 1)
    cze = np.zeros(nzl + 1)
    cdb = np.zeros(nzl + 1)
    lib().or_quad_table(len(zs), _d(zs), _d(ze), _d(db), zlatperi, zlatstrt, zlmin, dzl, nzl, _d(czs), _d(cze),
                        _d(cdb))
    return czs, cze, cdb


def sete_cond(conductors, phi, x, y, z, dx, dy, dz, xmmin, ymmin, zmmin, zgrid=0.0):
    """E at the particles with the conductor correction (lcorrectede) of
    sete3dwithconductor, efetch = 1; conductors is a finalized Conductors
    of the same grid. Returns new arrays ex, ey, ez (zero for particles
    outside the grid)."""
    nx, ny, nz = (s - 3 for s in phi.shape)
    phi = np.asfortranarray(phi, dtype=np.float64)
    n = len(x)
    ex, ey, ez = np.zeros(n), np.zeros(n), np.zeros(n)
    lib().or_sete_cond(conductors.h, nx, ny, nz, dx, dy, dz, xmmin, ymmin, zmmin, zgrid, _d(phi), n,
                       _d(np.ascontiguousarray(x, np.float64)), _d(np.ascontiguousarray(y, np.float64)),
                       _d(np.ascontiguousarray(z, np.float64)), _d(ex), _d(ey), _d(ez))
    return ex, ey, ez


_CENTERS = {"fullv": 0, "halfv": 1, "synchv": 2}


def push(p, ex, ey, ez, q, m, dt, tables, zlmin, dzl, zmmin, zmmax, prwall, prwallx=0.0, prwally=0.0,
         center="fullv"):
    """One padvnc3d advance (center "fullv", "halfv" or "synchv") of the
    particles in p, a dict of float64 arrays x,y,z,ux,uy,uz,gaminv
    (modified in place), with E already gathered into ex, ey, ez."""
    n = len(p["x"])
    if tables is None:
        czs = cze = cdb = None
        nzl = 0
    else:
        czs, cze, cdb = tables
        nzl = len(czs) - 1
    lib().or_push(_CENTERS[center], n, _d(p["x"]), _d(p["y"]), _d(p["z"]), _d(p["ux"]), _d(p["uy"]),
                  _d(p["uz"]), _d(p["gaminv"]), _d(ex), _d(ey), _d(ez), q, m, dt,
                  _d(czs) if czs is not None else None, _d(cze) if cze is not None else None,
                  _d(cdb) if cdb is not None else None, nzl, zlmin, dzl, zmmin, zmmax, prwall, prwallx, prwally)


def push_fullv(p, ex, ey, ez, q, m, dt, tables, zlmin, dzl, zmmin, zmmax, prwall, prwallx=0.0, prwally=0.0):
    """The fullv advance of push()."""
    push(p, ex, ey, ez, q, m, dt, tables, zlmin, dzl, zmmin, zmmax, prwall, prwallx, prwally, "fullv")


def zmoments(p, po, dt, zmmntmin, zmmntmax, nzmmnt, zbeam=0.0, dtscale=1.0, zmmntdtextmax=1e36):
    """getzmmnt moment sums (itask = 2, ifzmmnt = 2): p holds the particles
    (x, y, z, ux, uy, uz, gaminv), po the velocities ux, uy, uz a time dt
    earlier. Returns (zmmnts0[33], zmmnts[nzmmnt+1, 33])."""
    n = len(p["x"])
    z0 = np.zeros(33)
    zm = np.zeros((nzmmnt + 1, 33))
    lib().or_zmoments(n, *(_d(p[k]) for k in ("x", "y", "z", "ux", "uy", "uz", "gaminv")),
                      *(_d(po[k]) for k in ("ux", "uy", "uz")), dt, dtscale, zbeam, zmmntmin, zmmntmax, nzmmnt,
                      zmmntdtextmax, _d(z0), _d(zm))
    return z0, zm


def moments(p):
    out = np.zeros(8)
    lib().or_moments(len(p["x"]), _d(p["x"]), _d(p["y"]), _d(p["ux"]), _d(p["uy"]), _d(p["uz"]),
                     _d(p["gaminv"]), _d(out))
    return {"n": out[0], "xbar": out[1], "ybar": out[2], "xrms": out[3], "yrms": out[4], "epsx": out[5],
            "epsy": out[6]}


def ese(rho, phi, dx, dy, dz):
    """Field energy of getese3dfromrhophi (dw3d.F:708-777): rho (nx+1, ny+1,
    nz+1) and phi (nx+3, ny+3, nz+3), both Fortran-ordered."""
    rho = np.asfortranarray(rho, dtype=np.float64)
    phi = np.asfortranarray(phi, dtype=np.float64)
    nx, ny, nz = (n - 1 for n in rho.shape)
    return lib().or_ese(nx, ny, nz, _d(rho), _d(phi), dx, dy, dz)


def threads():
    """Host threads the oracle's parallel loops use (ORACLE_THREADS)."""
    return lib().or_threads()
