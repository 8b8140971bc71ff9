"""ctypes binding of libwarp_b200.so (include/warp_b200.h).

The library is the only compute path: if it is missing or cannot be loaded,
importing this module raises, there is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libwarp_b200.so")

WG_OK = 0
ERRORS = {
    -1: "WG_EINVAL", -2: "WG_ECUDA", -3: "WG_ESTATE", -4: "WG_EOVERFLOW", -5: "WG_ENODEV", -6: "WG_ENOMEM",
    -7: "WG_ETOOLARGE",
}


class WgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "WG_E?"), code, msg))
        self.code = code


class Grid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("xmmin", ctypes.c_double), ("xmmax", ctypes.c_double), ("ymmin", ctypes.c_double),
                ("ymmax", ctypes.c_double), ("zmmin", ctypes.c_double), ("zmmax", ctypes.c_double),
                ("bounds", ctypes.c_int * 6)]


class SolveOpts(ctypes.Structure):
    _fields_ = [("mgparam", ctypes.c_double), ("mgtol", ctypes.c_double), ("mgmaxiters", ctypes.c_int),
                ("mgmaxlevels", ctypes.c_int), ("downpasses", ctypes.c_int), ("uppasses", ctypes.c_int),
                ("lcndbndy", ctypes.c_int), ("precision", ctypes.c_int), ("tolkind", ctypes.c_int),
                ("flags", ctypes.c_int), ("mgmaxvcycles", ctypes.c_int)]


SOLVE_GRAPH, SOLVE_PDL = 1, 4


class SolveStats(ctypes.Structure):
    _fields_ = [("mgiters", ctypes.c_int), ("converged", ctypes.c_int), ("mgerror", ctypes.c_double),
                ("relres", ctypes.c_double)]


class Particles(ctypes.Structure):
    _fields_ = [("x", ctypes.c_void_p), ("y", ctypes.c_void_p), ("z", ctypes.c_void_p), ("ux", ctypes.c_void_p),
                ("uy", ctypes.c_void_p), ("uz", ctypes.c_void_p), ("gaminv", ctypes.c_void_p),
                ("np", ctypes.c_int64), ("q", ctypes.c_double), ("m", ctypes.c_double), ("w", ctypes.c_double)]


class ParticlesF32(ctypes.Structure):
    _fields_ = Particles._fields_


class PushParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("prwall", ctypes.c_double), ("prwallx", ctypes.c_double),
                ("prwally", ctypes.c_double), ("use_lattice", ctypes.c_int), ("center", ctypes.c_int)]


CENTER_FULLV, CENTER_HALFV, CENTER_SYNCHV = 0, 1, 2
CENTERS = {"fullv": CENTER_FULLV, "halfv": CENTER_HALFV, "synchv": CENTER_SYNCHV}


_c = ctypes
_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_i32p = ctypes.POINTER(ctypes.c_int32)
_i64p = ctypes.POINTER(ctypes.c_int64)

# name -> argtypes (all return int)
SIGNATURES = {
    "wg_create": [ctypes.POINTER(Grid), ctypes.POINTER(_vp)],
    "wg_destroy": [_vp],
    "wg_set_stream": [_vp, _vp],
    "wg_level_info": [_vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), _dp, ctypes.c_int],
    "wg_arrays": [_vp, ctypes.POINTER(_vp), ctypes.POINTER(_vp)],
    "wg_conductors_add_shape": [_vp, _c.c_int] + [_c.c_double] * 6 + [_c.c_int, _c.c_double],
    "wg_conductors_add_points": [_vp, _c.c_int, _c.c_int64, _i32p, _dp, _dp, _i32p],
    "wg_conductors_finalize": [_vp],
    "wg_conductors_clear": [_vp],
    "wg_conductors_counts": [_vp, _i64p],
    "wg_conductors_export": [_vp, _c.c_int, _i32p, _dp, _dp, _i32p],
    "wg_solve": [_vp, ctypes.POINTER(SolveOpts), ctypes.POINTER(SolveStats)],
    "wg_relresidual": [_vp, _c.c_double, _dp],
    "wg_residual_field": [_vp, _c.c_double, _vp],
    "wg_field_energy": [_vp, _dp],
    "wg_deposit": [_vp, ctypes.POINTER(Particles), _c.c_int],
    "wg_deposit_noalloc": [ctypes.POINTER(Grid), ctypes.POINTER(Particles), _vp, _c.c_int, _vp],
    "wg_finalize_rho": [_vp],
    "wg_fetch_e": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _c.c_int64],
    "wg_set_lattice": [_vp, _dp, _dp, _dp, _c.c_int, _c.c_double, _c.c_double],
    "wg_advance": [_vp, ctypes.POINTER(Particles), ctypes.POINTER(PushParams)],
    "wg_set_correctede": [_vp, _c.c_int],
    "wg_zmoments": [_vp, ctypes.POINTER(Particles), _vp, _vp, _vp] + [_c.c_double] * 5 + [_c.c_int, _c.c_double, _dp, _dp],
    "wg_deposit_begin": [_vp],
    "wg_deposit_add": [_vp, ctypes.POINTER(Particles)],
    "wg_deposit_end": [_vp, _c.c_int],
    "wg_moments": [_vp, ctypes.POINTER(Particles), _dp],
    "wg_prof_enable": [_vp, _c.c_int],
    "wg_prof_read": [_vp, _c.c_int, _dp, _i64p, _dp],
    "wg_launch_count": [_vp, _i64p],
    "wg_particle_keys": [_vp, ctypes.POINTER(Particles), _vp],
    "wg_particle_permute": [_vp, _vp, ctypes.POINTER(Particles), ctypes.POINTER(Particles)],
    "wg_deposit_f32": [_vp, ctypes.POINTER(ParticlesF32), _c.c_int],
    "wg_deposit_add_f32": [_vp, ctypes.POINTER(ParticlesF32)],
    "wg_advance_f32": [_vp, ctypes.POINTER(ParticlesF32), ctypes.POINTER(PushParams)],
    "wg_moments_f32": [_vp, ctypes.POINTER(ParticlesF32), _dp],
    "wg_advance_deposit": [_vp, ctypes.POINTER(Particles), ctypes.POINTER(PushParams)],
    "wg_advance_deposit_f32": [_vp, ctypes.POINTER(ParticlesF32), ctypes.POINTER(PushParams)],
    "wg_zmoments_f32": [_vp, ctypes.POINTER(ParticlesF32), _vp, _vp, _vp] + [_c.c_double] * 5 +
                       [_c.c_int, _c.c_double, _dp, _dp],
    "wg_particle_keys_f32": [_vp, ctypes.POINTER(ParticlesF32), _vp],
    "wg_particle_permute_f32": [_vp, _vp, ctypes.POINTER(ParticlesF32), ctypes.POINTER(ParticlesF32)],
    "wg_conv3_fwd": [_vp] + [_c.c_int] * 4 + [_vp, _vp, _c.c_int, _vp, _c.c_int, _c.c_int, _vp, _c.c_int, _c.c_int,
                     _vp, _vp],
    "wg_conv3_fwd_f32": [_vp] + [_c.c_int] * 4 + [_vp, _vp, _c.c_int, _vp, _c.c_int, _c.c_int, _vp, _c.c_int,
                         _c.c_int, _vp, _vp],
    "wg_conv3_wgrad": [_vp, _vp] + [_c.c_int] * 5 + [_vp, _vp, _c.c_int64, _vp, _vp],
    "wg_conv3_wgrad_scratch": [_c.c_int, _c.c_int, _i64p],
}

PROF_SOR0, PROF_DEPOSIT, PROF_ADVANCE, PROF_RESID0, PROF_RESTRICT0, PROF_EXPAND0, PROF_CORR = 0, 1, 2, 3, 4, 5, 6
PROF_COARSE = 7


def _load():
    if not os.path.exists(LIBPATH):
        raise ImportError("warp_b200: %s is missing; build it with `python -m warp_b200.build` "
                          "(there is no CPU fallback)" % LIBPATH)
    lib = ctypes.CDLL(LIBPATH)
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = ctypes.c_int
    lib.wg_last_error.restype = ctypes.c_char_p
    lib.wg_last_error.argtypes = []
    return lib


lib = _load()


def check(rc):
    if rc != WG_OK:
        raise WgError(rc, lib.wg_last_error().decode())
    return rc


def exported_symbols():
    """Names declared in include/warp_b200.h that the library exports."""
    return sorted(list(SIGNATURES) + ["wg_last_error"])
