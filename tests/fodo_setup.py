"""The FODO configuration of the reference's integration test
(warp_test/basicFODO_test.py): a matched 80 keV K+ beam (2 mA, 62.47 mm mrad)
in hard-edge quads (11 cm long, +-8.4818 T/m, half period 36 cm), on a
32 x 32 x 64 grid over one lattice period with periodic z and a 2 cm
absorbing pipe radius, 50 steps per period.

Shared by the envelope KAT, the long-run fixture generator and the long-run
GPU test. host_beam() draws the particles with torch's CPU generator, so the
oracle and the GPU start from the same bits."""
import math

import numpy as np

HLP, QUADLEN, DBDX, PIPERAD = 0.36, 0.11, 8.4817662372660610, 0.02
A0, B0, EMIT, IBEAM, EKIN = 15.60152892731585e-3, 8.75924684128793e-3, 62.46985327098694e-06, 2e-3, 80e3
NX, NY, NZ = 32, 32, 64
BOUNDS = (0, 0, 0, 0, 2, 2)
STEPS_PER_PERIOD = 50


def lattice():
    from warp_b200.lattice import Lattice, Quad
    return Lattice([Quad(-QUADLEN / 2, QUADLEN / 2, -DBDX), Quad(HLP - QUADLEN / 2, HLP + QUADLEN / 2, +DBDX)],
                   zlatperi=2 * HLP)


def species():
    """(q, m, v, gamma) of the K+ ions."""
    from warp_b200.constants import amu, clight, echarge
    m = 39.0983 * amu
    gamma = 1. + EKIN * echarge / (m * clight * clight)
    v = math.sqrt(1. - 1. / (gamma * gamma)) * clight
    return echarge, m, v, gamma


def envelope():
    """KV envelope (z, a, b, a', b') over one period from z = -HLP."""
    from warp_b200.envelope import integrate
    q, m, v, gamma = species()
    return integrate(lattice(), q, m, v, IBEAM, EMIT, EMIT, A0, B0, 0., 0., z0=-HLP, gamma=gamma)


def timestep():
    return (2 * HLP / STEPS_PER_PERIOD) / species()[2]


def weight(npart):
    q, m, v, _ = species()
    return IBEAM * (2 * HLP) / (q * v * npart)


def host_beam(npart, seed):
    """Matched semi-Gaussian beam as numpy arrays (x, y, z, ux, uy, uz, gaminv)."""
    import torch
    from warp_b200.particles import semigaussian_matched
    z, a, b, ap, bp = envelope()
    v = species()[2]
    gen = torch.Generator().manual_seed(seed)
    beam = semigaussian_matched(npart, gen, z, a, b, ap, bp, EMIT, EMIT, -HLP, HLP, v, device="cpu")
    return {k: np.ascontiguousarray(t.numpy()) for k, t in beam.items()}


def mesh():
    """(dx, dy, dz, xmmin, ymmin, zmmin)."""
    return 2 * PIPERAD / NX, 2 * PIPERAD / NY, 2 * HLP / NZ, -PIPERAD, -PIPERAD, -HLP


def quad_tables():
    """The lattice-cell tables MultiGridB200.setlattice installs (cells of dz
    from zmmin): (czs, cze, cdb, nzl, zlmin, dzl)."""
    dx, dy, dz, xmin, ymin, zmin = mesh()
    nzl = int(round((HLP - zmin) / dz)) + 1
    czs, cze, cdb = (np.ascontiguousarray(t) for t in lattice().tables(zmin, dz, nzl))
    return czs, cze, cdb, nzl, zmin, dz


def oracle_run(npart, nsteps, seed, mgtol, record_every=STEPS_PER_PERIOD):
    """The PIC run on the oracle: deposit + multigrid (max |dphi| <= mgtol)
    at load, then a halfv step and fullv steps, each followed by deposit and
    solve. Returns the V-cycles of every solve and, every record_every
    steps, the step, the emittances and the live-particle count."""
    from oracle import oracle
    q, m, v, _ = species()
    w = weight(npart)
    dx, dy, dz, xmin, ymin, zmin = mesh()
    czs, cze, cdb, nzl, zlmin, dzl = quad_tables()
    p = host_beam(npart, seed)
    phi = np.zeros((NX + 3, NY + 3, NZ + 3), order="F")

    def solve():
        rho = np.zeros((NX + 1, NY + 1, NZ + 1), order="F")
        oracle.setrho(rho, p["x"], p["y"], p["z"], q, w, dx, dy, dz, xmin, ymin, zmin, gaminv=p["gaminv"])
        oracle.rhobc(rho, BOUNDS)
        return oracle.mgsolve(phi, rho, dx, dy, dz, BOUNDS, mgtol=mgtol)[0]

    dt = timestep()
    vcycles = [solve()]
    rec = []
    for n in range(nsteps):
        ex, ey, ez = oracle.sete(phi, p["x"], p["y"], p["z"], dx, dy, dz, xmin, ymin, zmin)
        oracle.push(p, ex, ey, ez, q, m, dt, (czs, cze, cdb), zlmin, dzl, zmin, HLP, PIPERAD,
                    center="halfv" if n == 0 else "fullv")
        vcycles.append(solve())
        if (n + 1) % record_every == 0:
            mo = oracle.moments(p)
            rec.append((n + 1, mo["epsx"], mo["epsy"], mo["n"]))
    r = np.array(rec)
    return {"step": r[:, 0].astype(np.int64), "epsx": r[:, 1], "epsy": r[:, 2], "live": r[:, 3].astype(np.int64),
            "vcycles": np.array(vcycles, dtype=np.int32)}
