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
