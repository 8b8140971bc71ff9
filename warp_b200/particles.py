"""Device-resident particle group (the role of top.pgroup) and the seeded
semi-Gaussian beam loader used for the synthetic workloads.

Arrays are torch tensors on the CUDA device (SoA: x, y, z, ux, uy, uz,
gaminv, and ex, ey, ez for fetche). The particle arrays are float64, the
reference's storage, or float32 for the mixed-precision form whose push runs
in FP32 (dtype=torch.float32; the library's _f32 entry points); ex, ey, ez
stay float64. A lost particle has gaminv == 0, the stckxy3d convention
(pywarp90/w3d.F:11520-11535); lost particles are skipped by the deposit,
push and moments kernels.
"""
import math

import numpy as np
import torch

from . import _lib
from .constants import clight, echarge, proton_mass
from .workloads import beam_weight, semigaussian  # noqa: F401

FIELDS = ("x", "y", "z", "ux", "uy", "uz", "gaminv")


class ParticleGroup:
    def __init__(self, arrays, q=echarge, m=proton_mass, w=1.0, device="cuda", with_fields=True,
                 dtype=torch.float64):
        """arrays: dict of equal-length 1-D arrays (numpy or torch) for
        FIELDS, stored as `dtype` (torch.float64 or torch.float32)."""
        if dtype not in (torch.float64, torch.float32):
            raise ValueError("ParticleGroup: dtype must be torch.float64 or torch.float32")
        self.dtype = dtype
        self.q, self.m, self.w = float(q), float(m), float(w)
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        n = len(arrays["x"])
        for f in FIELDS:
            a = arrays[f]
            t = torch.as_tensor(a).to(device=self.device, dtype=dtype).contiguous()
            if t.shape != (n,):
                raise ValueError("particle array %s has shape %s, expected (%d,)" % (f, tuple(t.shape), n))
            setattr(self, f, t)
        if with_fields:
            self.ex = torch.zeros(n, dtype=torch.float64, device=self.device)
            self.ey = torch.zeros_like(self.ex)
            self.ez = torch.zeros_like(self.ex)
        self._struct = None

    @property
    def np(self):
        return int(self.x.shape[0])

    @property
    def fp32(self):
        return self.dtype == torch.float32

    def fn(self, name):
        """The library entry point `name` for this group's storage (the _f32
        form for FP32 particles)."""
        return getattr(_lib.lib, name + "_f32" if self.fp32 else name)

    def cstruct(self, start=0, stop=None):
        """C view of particles start..stop-1 (all by default): a
        wg_particles, or a wg_particles_f32 for FP32 storage."""
        stop = self.np if stop is None else int(stop)
        s = _lib.ParticlesF32() if self.fp32 else _lib.Particles()
        size = 4 if self.fp32 else 8
        for f in FIELDS:
            setattr(s, f, getattr(self, f).data_ptr() + size * int(start))
        s.np = stop - int(start)
        s.q, s.m, s.w = self.q, self.m, self.w
        return s

    def sort(self, solver, compact=True):
        """Sorts the particles by cell of the solver's grid
        (particlesortxyzwithcopy, pywarp90/top.F:5095): keys from the
        library, a stable sort of the keys, one permutation kernel over the
        7 arrays. Lost particles (gaminv == 0) end up at the back; with
        compact=True they are dropped. Order within a cell keeps the old
        order, so the result is deterministic."""
        import ctypes
        n = self.np
        if n == 0:
            return
        keys = torch.empty(n, dtype=torch.int64, device=self.device)
        s = self.cstruct()
        _lib.check(self.fn("wg_particle_keys")(solver._h, ctypes.byref(s), ctypes.c_void_p(keys.data_ptr())))
        sentinel = (solver.nx + 1) * (solver.ny + 1) * (solver.nz + 1)
        if sentinel < 2 ** 31:
            # 32-bit keys: half the radix passes of the 64-bit sort
            keys = keys.to(torch.int32)
        perm = torch.argsort(keys, stable=True)
        nlive = n
        if compact:
            nlive = int(torch.searchsorted(keys[perm], torch.tensor([sentinel], device=self.device,
                                                                     dtype=keys.dtype)).item())
        new = {f: torch.empty(nlive, dtype=self.dtype, device=self.device) for f in FIELDS}
        d = _lib.ParticlesF32() if self.fp32 else _lib.Particles()
        for f in FIELDS:
            setattr(d, f, new[f].data_ptr())
        d.np = nlive
        s.np = nlive
        d.q, d.m, d.w = self.q, self.m, self.w
        _lib.check(self.fn("wg_particle_permute")(solver._h, ctypes.c_void_p(perm.data_ptr()), ctypes.byref(s),
                                                  ctypes.byref(d)))
        for f in FIELDS:
            setattr(self, f, new[f])
        if hasattr(self, "ex") and self.ex.shape[0] != nlive:
            self.ex = torch.zeros(nlive, dtype=torch.float64, device=self.device)
            self.ey = torch.zeros_like(self.ex)
            self.ez = torch.zeros_like(self.ex)

    def to_numpy(self):
        return {f: getattr(self, f).cpu().numpy() for f in FIELDS}

    def nlive(self):
        return int((self.gaminv != 0).sum().item())


def semigaussian_device(n, generator, radius=2e-3, mismatch=0.0, angle_rms=5e-3, zmin=0.0, zmax=1.0,
                        ekin_ev=1e6, mass=proton_mass, device="cuda"):
    """semigaussian() drawn on the device from a seeded torch.Generator (used
    to generate many training beams quickly). Returns a dict of tensors."""
    gamma = 1. + ekin_ev * echarge / (mass * clight * clight)
    vz = math.sqrt(1. - 1. / (gamma * gamma)) * clight
    kw = dict(generator=generator, device=device, dtype=torch.float64)
    r = torch.sqrt(torch.rand(n, **kw))
    th = 2. * math.pi * torch.rand(n, **kw)
    x = radius * (1. + mismatch) * r * torch.cos(th)
    y = radius * (1. - mismatch) * r * torch.sin(th)
    z = zmin + (zmax - zmin) * torch.rand(n, **kw)
    ux = angle_rms * torch.randn(n, **kw) * vz
    uy = angle_rms * torch.randn(n, **kw) * vz
    return {"x": x, "y": y, "z": z, "ux": ux, "uy": uy, "uz": torch.full((n,), vz, **{k: kw[k] for k in ("device", "dtype")}),
            "gaminv": torch.ones(n, device=device, dtype=torch.float64)}


def semigaussian_matched(n, generator, z, a, b, ap, bp, emitx, emity, zmin, zmax, v, device="cuda"):
    """Semi-Gaussian beam that follows an envelope, as the reference loads
    it from its env package (w3d.distrbtn = "semigaus"): z uniform in
    [zmin, zmax); at each particle's z the envelope (a, b, a', b', given on
    the grid z and interpolated linearly) sets a uniform density in the
    ellipse (x/a)^2 + (y/b)^2 <= 1, the slope x' = (a'/a) x plus a Gaussian
    spread of rms emitx / (2 a) (so the 4 x rms emittance is emitx), and
    likewise in y. uz = v (non-relativistic, gaminv = 1)."""
    kw = dict(generator=generator, device=device, dtype=torch.float64)
    zt = torch.as_tensor(np.asarray(z, dtype=np.float64), device=device)

    def interp(f):
        ft = torch.as_tensor(np.asarray(f, dtype=np.float64), device=device)
        idx = torch.clamp(torch.searchsorted(zt, zp) - 1, 0, zt.numel() - 2)
        t = (zp - zt[idx]) / (zt[idx + 1] - zt[idx])
        return ft[idx] + t * (ft[idx + 1] - ft[idx])

    zp = zmin + (zmax - zmin) * torch.rand(n, **kw)
    aa, bb, aap, bbp = interp(a), interp(b), interp(ap), interp(bp)
    r = torch.sqrt(torch.rand(n, **kw))
    th = 2. * math.pi * torch.rand(n, **kw)
    x = aa * r * torch.cos(th)
    y = bb * r * torch.sin(th)
    xp = aap / aa * x + emitx / (2. * aa) * torch.randn(n, **kw)
    yp = bbp / bb * y + emity / (2. * bb) * torch.randn(n, **kw)
    return {"x": x, "y": y, "z": zp, "ux": xp * v, "uy": yp * v,
            "uz": torch.full((n,), float(v), device=device, dtype=torch.float64),
            "gaminv": torch.ones(n, device=device, dtype=torch.float64)}


def rms_along_z(pgroup, zmin, zmax, nz, periodic=True):
    """rms x and y sizes of the live particles on the z grid nodes
    zmin + k (zmax - zmin) / nz, k = 0..nz, with linear weighting in z (the
    z moments of getzmmnt, top.F:521-1444, xrmsz and yrmsz). With periodic z
    the end nodes share their particles. Returns two numpy arrays."""
    import torch as _t
    live = pgroup.gaminv != 0
    x, y, z = pgroup.x[live], pgroup.y[live], pgroup.z[live]
    dz = (zmax - zmin) / nz
    s = (z - zmin) / dz
    k = _t.clamp(_t.floor(s).long(), 0, nz - 1)
    f = s - k
    n0 = _t.zeros(nz + 1, dtype=_t.float64, device=x.device)
    sums = [n0.clone() for _ in range(5)]
    for arr, val in zip(sums, (_t.ones_like(x), x, y, x * x, y * y)):
        arr.index_add_(0, k, (1. - f) * val)
        arr.index_add_(0, k + 1, f * val)
    if periodic:
        for arr in sums:
            arr[0] += arr[nz]
            arr[nz] = arr[0]
    w, sx, sy, sxx, syy = sums
    w = _t.clamp(w, min=1e-300)
    xr = _t.sqrt(_t.clamp(sxx / w - (sx / w) ** 2, min=0.))
    yr = _t.sqrt(_t.clamp(syy / w - (sy / w) ** 2, min=0.))
    return xr.cpu().numpy(), yr.cpu().numpy()
