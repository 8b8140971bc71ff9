"""Manufactured-solution harness of the reference's multigrid known-answer
test, restated: warp_test/MutltiGrid3D_test.py:15-83 with
warp_test/fieldsolvertesttools.py:4-127.

phi_exact = sin(pi x + .5) sin(2 pi y + 2.5) sin(pi z + 1.111) on a 24x22x18
cell grid over [-1,1]^3; rho is the DISCRETE 7-point Laplacian of phi_exact
(times -eps0) with guard values set the way the solver sets them for each
boundary type, so the exact discrete solution is known.
"""
import itertools

import numpy as np

NX, NY, NZ = 24, 22, 18
XMIN, XMAX = -1.0, 1.0


def mesh():
    dx = (XMAX - XMIN) / NX
    dy = (XMAX - XMIN) / NY
    dz = (XMAX - XMIN) / NZ
    x = XMIN - dx + dx * np.arange(NX + 3)
    y = XMIN - dy + dy * np.arange(NY + 3)
    z = XMIN - dz + dz * np.arange(NZ + 3)
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    return dx, dy, dz, X, Y, Z


def testphi():
    dx, dy, dz, X, Y, Z = mesh()
    return np.asfortranarray(np.sin(np.pi * X + 0.5) * np.sin(2 * np.pi * Y + 2.5) * np.sin(np.pi * Z + 1.111))


def boundary_combos():
    """All boundary combinations of the reference test, deduplicated, in its
    loop order (periodic on one side forces periodic on the other)."""
    seen = []
    for zp, zm, yp, ym, xp, xm in itertools.product([0, 1, 2], repeat=6):
        if zp == 2: zm = 2
        if zm == 2: zp = 2
        if yp == 2: ym = 2
        if ym == 2: yp = 2
        if xp == 2: xm = 2
        if xm == 2: xp = 2
        b = (xm, xp, ym, yp, zm, zp)
        if b not in seen:
            seen.append(b)
    return seen


def gettestrho(phi, bounds, eps0):
    """fieldsolvertesttools.gettestrho (serial)."""
    dx, dy, dz, *_ = mesh()
    phi = phi.copy(order="F")
    c = slice(1, -1)
    lb = bounds
    if lb[0] == 1: phi[0, c, c] = phi[2, c, c]
    if lb[1] == 1: phi[-1, c, c] = phi[-3, c, c]
    if lb[2] == 1: phi[c, 0, c] = phi[c, 2, c]
    if lb[3] == 1: phi[c, -1, c] = phi[c, -3, c]
    if lb[4] == 1: phi[c, c, 0] = phi[c, c, 2]
    if lb[5] == 1: phi[c, c, -1] = phi[c, c, -3]
    if lb[0] == 0: phi[0, c, c] = 2. * phi[1, c, c] - phi[2, c, c]
    if lb[1] == 0: phi[-1, c, c] = 2. * phi[-2, c, c] - phi[-3, c, c]
    if lb[2] == 0: phi[c, 0, c] = 2. * phi[c, 1, c] - phi[c, 2, c]
    if lb[3] == 0: phi[c, -1, c] = 2. * phi[c, -2, c] - phi[c, -3, c]
    if lb[4] == 0: phi[c, c, 0] = 2. * phi[c, c, 1] - phi[c, c, 2]
    if lb[5] == 0: phi[c, c, -1] = 2. * phi[c, c, -2] - phi[c, c, -3]
    rho = -eps0 * ((phi[:-2, c, c] - 2. * phi[c, c, c] + phi[2:, c, c]) / dx ** 2 +
                   (phi[c, :-2, c] - 2. * phi[c, c, c] + phi[c, 2:, c]) / dy ** 2 +
                   (phi[c, c, :-2] - 2. * phi[c, c, c] + phi[c, c, 2:]) / dz ** 2)
    return np.asfortranarray(rho), phi


def clearcorners(phi):
    phi[0, 0, :] = 0.
    phi[0, -1, :] = 0.
    phi[0, :, 0] = 0.
    phi[0, :, -1] = 0.
    phi[-1, 0, :] = 0.
    phi[-1, -1, :] = 0.
    phi[-1, :, 0] = 0.
    phi[-1, :, -1] = 0.
    phi[:, 0, 0] = 0.
    phi[:, 0, -1] = 0.
    phi[:, -1, 0] = 0.
    phi[:, -1, -1] = 0.


def setup(bounds, eps0):
    """Returns (rho, phi_initial, phi_expected) as fieldsolvertesttools does
    before the solve."""
    rho, phi = gettestrho(testphi(), bounds, eps0)
    sphi = np.zeros_like(phi, order="F")
    if bounds[0] == 0: sphi[1, :, :] = phi[1, :, :]
    if bounds[1] == 0: sphi[-2, :, :] = phi[-2, :, :]
    if bounds[2] == 0: sphi[:, 1, :] = phi[:, 1, :]
    if bounds[3] == 0: sphi[:, -2, :] = phi[:, -2, :]
    if bounds[4] == 0: sphi[:, :, 1] = phi[:, :, 1]
    if bounds[5] == 0: sphi[:, :, -2] = phi[:, :, -2]
    return rho, sphi, phi


def error(solved, expected, bounds):
    """The error measure of fieldsolvertesttools (after the solve)."""
    solved = solved.copy(order="F")
    expected = expected.copy(order="F")
    if 0 not in bounds:
        c = slice(1, -1)
        solved -= solved[c, c, c].mean()
        expected -= expected[c, c, c].mean()
    clearcorners(expected)
    clearcorners(solved)
    return float(np.max(np.abs(solved - expected)))
