"""Device-resident particle group (the role of top.pgroup) and the seeded
semi-Gaussian beam loader used for the synthetic workloads.

Arrays are float64 torch tensors on the CUDA device (SoA: x, y, z, ux, uy,
uz, gaminv, ex, ey, ez). A lost particle has gaminv == 0, the stckxy3d
convention (pywarp90/w3d.F:11520-11535); lost particles are skipped by the
deposit, push and moments kernels.
"""
import math

import numpy as np
import torch

from . import _lib
from .constants import clight, echarge, proton_mass

FIELDS = ("x", "y", "z", "ux", "uy", "uz", "gaminv")


class ParticleGroup:
    def __init__(self, arrays, q=echarge, m=proton_mass, w=1.0, device="cuda", with_fields=True):
        """arrays: dict of equal-length 1-D arrays (numpy or torch) for FIELDS."""
        self.q, self.m, self.w = float(q), float(m), float(w)
        self.device = torch.device(device)
        if self.device.type == "cuda" and self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        n = len(arrays["x"])
        for f in FIELDS:
            a = arrays[f]
            t = torch.as_tensor(a, dtype=torch.float64).to(self.device).contiguous()
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

    def cstruct(self, start=0, stop=None):
        """C view of particles start..stop-1 (all by default)."""
        stop = self.np if stop is None else int(stop)
        s = _lib.Particles()
        for f in FIELDS:
            setattr(s, f, getattr(self, f).data_ptr() + 8 * int(start))
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
        _lib.check(_lib.lib.wg_particle_keys(solver._h, ctypes.byref(s), ctypes.c_void_p(keys.data_ptr())))
        perm = torch.argsort(keys, stable=True)
        nlive = n
        if compact:
            sentinel = (solver.nx + 1) * (solver.ny + 1) * (solver.nz + 1)
            nlive = int(torch.searchsorted(keys[perm], torch.tensor([sentinel], device=self.device)).item())
        new = {f: torch.empty(nlive, dtype=torch.float64, device=self.device) for f in FIELDS}
        d = _lib.Particles()
        for f in FIELDS:
            setattr(d, f, new[f].data_ptr())
        d.np = nlive
        s.np = nlive
        d.q, d.m, d.w = self.q, self.m, self.w
        _lib.check(_lib.lib.wg_particle_permute(solver._h, ctypes.c_void_p(perm.data_ptr()), ctypes.byref(s),
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


def semigaussian(n, seed=0, radius=2e-3, mismatch=0.0, angle_rms=5e-3, zmin=0.0, zmax=1.0, ekin_ev=1e6,
                 mass=proton_mass, xcent=0.0, ycent=0.0):
    """Seeded semi-Gaussian beam: uniform in an ellipse with semi-axes
    radius*(1+mismatch) (x) and radius*(1-mismatch) (y), Gaussian transverse
    angles of rms `angle_rms` (x' = ux/uz), uniform in z. Non-relativistic
    push (lrelativ = false): gaminv = 1, uz = beta*c. Returns numpy arrays.
    Philox counter-based generator, so the stream is reproducible."""
    rng = np.random.Generator(np.random.Philox(seed))
    gamma = 1. + ekin_ev * echarge / (mass * clight * clight)
    beta = math.sqrt(1. - 1. / (gamma * gamma))
    vz = beta * clight
    r = np.sqrt(rng.random(n))
    th = 2. * np.pi * rng.random(n)
    ax, ay = radius * (1. + mismatch), radius * (1. - mismatch)
    x = xcent + ax * r * np.cos(th)
    y = ycent + ay * r * np.sin(th)
    z = zmin + (zmax - zmin) * rng.random(n)
    xp = angle_rms * rng.standard_normal(n)
    yp = angle_rms * rng.standard_normal(n)
    uz = np.full(n, vz)
    return {"x": x, "y": y, "z": z, "ux": xp * vz, "uy": yp * vz, "uz": uz, "gaminv": np.ones(n)}


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


def beam_weight(current, length, n, ekin_ev=1e6, mass=proton_mass, charge=echarge):
    """Real particles per macroparticle for a beam of `current` (A) filling
    `length` (m): w = I L / (q v N)."""
    gamma = 1. + ekin_ev * echarge / (mass * clight * clight)
    v = math.sqrt(1. - 1. / (gamma * gamma)) * clight
    return current * length / (charge * v * n)
