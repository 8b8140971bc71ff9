"""Synthetic workloads of the PIC step (mesh, beam, lattice and conductor
parameters) and the seeded beam loader, as plain data and numpy: nothing here
loads the CUDA library, so the CPU reference timing can use it too.

Workloads:
  A: 32x32x64 cells over 8 cm x 8 cm x 1 m, 2e5 protons at 1 MeV,
      semi-Gaussian (2 mm radius, 5 mrad rms angle, 10 mA), FODO of
      hard-edge quads 10 cm long at +-15 T/m with 50 cm period, grounded pipe
      of radius 3.5 cm, periodic z, 50 steps.
  B: the same physics on 256x256x512 cells with 5e7 particles, 4 mm radius
      with 20% envelope mismatch, 1000 steps.
  D: the box of B on 128x128x256 cells (training grid of the learned warm
      start).
  E: 256x256x1024 cells, 2e8 particles, plus four electrostatic quadrupole
      rods (radius 1 cm, +-20 kV) inside the pipe.
"""
import math

import numpy as np

from .constants import clight, echarge, proton_mass

WORKLOADS = {
    "A": dict(nx=32, ny=32, nz=64, npart=200_000, radius=2e-3, mismatch=0.0, nsteps=50, rods=False),
    "B": dict(nx=256, ny=256, nz=512, npart=50_000_000, radius=4e-3, mismatch=0.2, nsteps=1000, rods=False),
    "E": dict(nx=256, ny=256, nz=1024, npart=200_000_000, radius=4e-3, mismatch=0.2, nsteps=1000, rods=True),
    # the box of B at half resolution: training grid of the learned warm start;
    # 5e7 particles give the same particles per cell as B's beam seen on this
    # grid (B restricted by two), where the network is applied
    "D": dict(nx=128, ny=128, nz=256, npart=50_000_000, radius=4e-3, mismatch=0.2, nsteps=8, rods=False),
}

COMMON = dict(xmmin=-0.04, xmmax=0.04, ymmin=-0.04, ymmax=0.04, zmmin=0.0, zmmax=1.0, ekin_ev=1.0e6,
              angle_rms=5e-3, current=10e-3, quad_gradient=15.0, quad_length=0.10, period=0.50,
              pipe_radius=0.035, rod_radius=0.01, rod_voltage=20e3, rod_center=0.0225, seed=0,
              steps_per_period=50)


def workload(name, **over):
    cfg = dict(COMMON)
    cfg.update(WORKLOADS[name])
    cfg.update(over)
    cfg["name"] = name
    return cfg


def beam_velocity(cfg):
    gamma = 1. + cfg["ekin_ev"] * echarge / (proton_mass * clight * clight)
    return math.sqrt(1. - 1. / (gamma * gamma)) * clight


def timestep(cfg):
    return (cfg["period"] / cfg["steps_per_period"]) / beam_velocity(cfg)



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


def beam_weight(current, length, n, ekin_ev=1e6, mass=proton_mass, charge=echarge):
    """Real particles per macroparticle for a beam of `current` (A) filling
    `length` (m): w = I L / (q v N)."""
    gamma = 1. + ekin_ev * echarge / (mass * clight * clight)
    v = math.sqrt(1. - 1. / (gamma * gamma)) * clight
    return current * length / (charge * v * n)


# Config C: the standalone multigrid solve on a 512^3 grid over the unit
# cube, Dirichlet on every face; rho a sum of 64 seeded Gaussian blobs (sigma
# 2-20 cells, amplitudes uniform in [-1, 1]); conductors a grounded cylinder
# and 8 spheres at seeded potentials in [-1, 1] V; solved to a 1e-10 relative
# residual.
CONFIG_C = dict(n=512, nblob=64, blob_seed=7, shape_seed=2024, mgtol=1e-10)


def config_c_shapes(seed=CONFIG_C["shape_seed"]):
    """The grounded cylinder and 8 spheres of config C (conductors module
    shapes, unit cube)."""
    from . import conductors as C
    rng = np.random.default_rng(seed)
    shapes = [C.ZCylinderOut(radius=0.45, length=10.0, voltage=0.0, xcent=0.5, ycent=0.5, zcent=0.5)]
    for _ in range(8):
        r = rng.uniform(0.03, 0.06)
        ang, rad = rng.uniform(0, 2 * math.pi), rng.uniform(0, 0.3)
        shapes.append(C.Sphere(radius=r, voltage=rng.uniform(-1, 1), xcent=0.5 + rad * math.cos(ang),
                               ycent=0.5 + rad * math.sin(ang), zcent=rng.uniform(0.2, 0.8)))
    return shapes


def blobs_rho(solver, nblob, seed, scale):
    """Sum of seeded Gaussian blobs (sigma 2-20 cells, amplitude U[-1,1])
    times `scale`, written into solver.rho on its device from separable 1-D
    factors."""
    import torch
    rng = np.random.default_rng(seed)
    dev = solver.device
    x = torch.linspace(solver.xmmin, solver.xmmax, solver.nx + 1, device=dev, dtype=torch.float64)
    y = torch.linspace(solver.ymmin, solver.ymmax, solver.ny + 1, device=dev, dtype=torch.float64)
    z = torch.linspace(solver.zmmin, solver.zmmax, solver.nz + 1, device=dev, dtype=torch.float64)
    rho = torch.zeros((solver.nx + 1, solver.ny + 1, solver.nz + 1), dtype=torch.float64, device=dev)
    for _ in range(nblob):
        c = [rng.uniform(lo + 0.2 * (hi - lo), hi - 0.2 * (hi - lo)) for lo, hi in
             ((solver.xmmin, solver.xmmax), (solver.ymmin, solver.ymmax), (solver.zmmin, solver.zmmax))]
        sig = rng.uniform(2, 20) * solver.dx
        amp = rng.uniform(-1, 1)
        gx = torch.exp(-(x - c[0]) ** 2 / (2 * sig * sig))
        gy = torch.exp(-(y - c[1]) ** 2 / (2 * sig * sig))
        gz = torch.exp(-(z - c[2]) ** 2 / (2 * sig * sig))
        rho += amp * gx[:, None, None] * gy[None, :, None] * gz[None, None, :]
    solver.rho.copy_(rho * scale)
