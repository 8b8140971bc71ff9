"""KV envelope equations of a beam in a hard-edge quadrupole lattice: the
matched-beam reference that the reference's integration test
(warp_test/basicFODO_test.py) compares the PIC rms envelope against. The
reference computes it with its env package, which is not part of this
build; this module integrates the same equations:

    a'' + kappa(z) a - 2 Q / (a + b) - emitx^2 / a^3 = 0
    b'' - kappa(z) b - 2 Q / (a + b) - emity^2 / b^3 = 0

a and b are the edge radii (twice the rms sizes), emitx and emity the edge
(4 x rms) emittances, Q = q I / (2 pi eps0 m gamma^3 v^3) the perveance,
and kappa = q db / (gamma m v) the focusing strength of a magnetic quad of
gradient db (T/m). Inside a quad db > 0 focuses in x for q > 0, as in the
particle push.

The integration is classical fourth-order Runge-Kutta, restarted at every
quad edge so that the hard-edge steps are exact.
"""
import math

import numpy as np

from .constants import eps0


def perveance(q, m, current, v, gamma=1.0):
    return q * current / (2.0 * math.pi * eps0 * m * gamma ** 3 * v ** 3)


def _kappa_at(lattice, q, m, v, gamma, z):
    """Focusing strength at z (periodic lattice)."""
    P = lattice.zlatperi
    zl = (z - lattice.zlatstrt) % P + lattice.zlatstrt
    for quad in lattice.quads:
        for shift in (-P, 0.0, P):
            if quad.zs + shift <= zl < quad.ze + shift:
                return q * quad.db / (gamma * m * v)
    return 0.0


def _edges(lattice, z0, z1):
    """Quad edges strictly inside (z0, z1)."""
    P = lattice.zlatperi
    out = []
    k0 = math.floor((z0 - lattice.zlatstrt) / P) - 1
    k1 = math.ceil((z1 - lattice.zlatstrt) / P) + 1
    for k in range(k0, k1 + 1):
        for quad in lattice.quads:
            for e in (quad.zs, quad.ze):
                z = e + k * P
                if z0 < z < z1:
                    out.append(z)
    return sorted(set(out))


def integrate(lattice, q, m, v, current, emitx, emity, a0, b0, ap0=0.0, bp0=0.0, z0=0.0, z1=None, dz=1e-4,
              gamma=1.0):
    """Envelope from z0 to z1 (default one lattice period). Returns arrays
    z, a, b, ap, bp at about dz spacing, with every quad edge included."""
    if z1 is None:
        z1 = z0 + lattice.zlatperi
    Q = perveance(q, m, current, v, gamma)
    pts = [z0] + _edges(lattice, z0, z1) + [z1]

    def rhs(kap, y):
        a, b, ap, bp = y
        return np.array([ap, bp, -kap * a + 2.0 * Q / (a + b) + emitx ** 2 / a ** 3,
                         kap * b + 2.0 * Q / (a + b) + emity ** 2 / b ** 3])

    y = np.array([a0, b0, ap0, bp0], dtype=np.float64)
    zs, ys = [z0], [y.copy()]
    for za, zb in zip(pts[:-1], pts[1:]):
        kap = _kappa_at(lattice, q, m, v, gamma, 0.5 * (za + zb))
        n = max(1, int(math.ceil((zb - za) / dz)))
        h = (zb - za) / n
        z = za
        for _ in range(n):
            k1 = rhs(kap, y)
            k2 = rhs(kap, y + 0.5 * h * k1)
            k3 = rhs(kap, y + 0.5 * h * k2)
            k4 = rhs(kap, y + h * k3)
            y = y + (h / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
            z += h
            zs.append(z)
            ys.append(y.copy())
    ys = np.array(ys)
    return np.array(zs), ys[:, 0], ys[:, 1], ys[:, 2], ys[:, 3]


def undepressed_phase_advance(lattice, q, m, v, gamma=1.0, z0=0.0):
    """Single-particle phase advance per period in x (degrees), from the
    hard-edge transfer matrices of one period."""
    P = lattice.zlatperi
    pts = [z0] + _edges(lattice, z0, z0 + P) + [z0 + P]
    M = np.eye(2)
    for za, zb in zip(pts[:-1], pts[1:]):
        L = zb - za
        k = _kappa_at(lattice, q, m, v, gamma, 0.5 * (za + zb))
        if k > 0:
            s = math.sqrt(k)
            T = np.array([[math.cos(s * L), math.sin(s * L) / s], [-s * math.sin(s * L), math.cos(s * L)]])
        elif k < 0:
            s = math.sqrt(-k)
            T = np.array([[math.cosh(s * L), math.sinh(s * L) / s], [s * math.sinh(s * L), math.cosh(s * L)]])
        else:
            T = np.array([[1.0, L], [0.0, 1.0]])
        M = T @ M
    c = 0.5 * np.trace(M)
    if abs(c) > 1:
        raise ValueError("lattice is unstable (|cos sigma0| > 1)")
    return math.degrees(math.acos(c))


def depressed_phase_advance(z, a, emit):
    """Phase advance of the matched envelope per period (degrees):
    sigma = integral of emit / a^2 dz (trapezoid rule)."""
    return math.degrees(np.trapezoid(emit / a ** 2, z))
