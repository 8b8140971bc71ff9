"""A long run against the oracle: the FODO beam of the reference's
integration test (tests/fodo_setup.py; 20000 particles, 32 x 32 x 64 cells,
multigrid to max |dphi| <= 1e-6 V) over 1000 steps, 20 lattice periods,
compared period by period with the oracle's run stored in
tests/golden/fodo_long_run.npz (made by tests/golden/make_fodo_long_run.py).

- Plain FP64 form: the emittances within 1e-9 relative of the oracle's at
  every period, the same live-particle counts, and the same V-cycle count
  in all but at most two of the 1001 solves. Over 1000 steps the only
  difference is the 2^-46 fixed-point rounding of the deposit.
- Mixed form (FP32 V-cycles inside FP64 defect correction, FP32 particles
  with an FP32 push): the emittances within 1e-4 relative of the FP64
  oracle after 1000 steps, the stated accuracy target of the mixed form,
  and at most two particles lost differently. Its final phi and grid E
  (centred differences) are within 1e-4 of max|.| of the plain run's, and
  the particles' final positions and transverse velocities within 1e-4 of
  the plain run's rms values (rms of the differences). The plain run
  stands in for the oracle here: it matches the fixture's emittances
  within 1e-9 with the same V-cycle counts.

On the oracle the run responds linearly to small changes of the field: a
1e-8 relative change of rho moves the emittance by about 1e-8 after 1000
steps, so differences do not grow exponentially here."""
import os

import numpy as np
import pytest
import torch

from tests import fodo_setup as F

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fodo_long_run.npz")


def _run(precision, g):
    from warp_b200.multigrid import MultiGridB200
    from warp_b200.particles import ParticleGroup
    dtype = torch.float32 if precision == "mixed" else torch.float64
    q, m, v, _ = F.species()
    npart = int(g["npart"])
    p = F.host_beam(npart, int(g["seed"]))
    assert np.array_equal(p["x"][:8], g["x0"]), "the CPU generator no longer draws the fixture's particles"
    dx, dy, dz, xmin, ymin, zmin = F.mesh()
    s = MultiGridB200(F.NX, F.NY, F.NZ, xmin, -xmin, ymin, -ymin, zmin, -zmin, bounds=F.BOUNDS,
                      precision=precision, tolkind="mgerror", mgtol=float(g["mgtol"]), mgverbose=-1)
    s.setlattice(F.lattice())
    pg = ParticleGroup(p, q=q, m=m, w=F.weight(npart), dtype=dtype)
    s.addpgroup(pg)
    s.loadrho()
    s.solve()
    vcycles = [s.mgiters]
    dt = F.timestep()
    every = int(g["step"][0])
    rec = []
    for n in range(int(g["nsteps"])):
        s.advance(pg, dt, prwall=F.PIPERAD, center="halfv" if n == 0 else "fullv")
        s.loadrho()
        s.solve()
        assert s.converged, "step %d" % n
        vcycles.append(s.mgiters)
        if (n + 1) % every == 0:
            mo = s.moments(pg)
            rec.append((mo["epsx"], mo["epsy"], mo["n"]))
    r = np.array(rec)
    parts = {k: v.astype(np.float64) for k, v in pg.to_numpy().items()}
    return r[:, 0], r[:, 1], r[:, 2].astype(np.int64), np.array(vcycles), s.phi.cpu().numpy(), parts


def _efield(phi):
    """E = -grad phi by centred differences on the nodes 0..n."""
    dx, dy, dz, *_ = F.mesh()
    return (-(phi[2:, 1:-1, 1:-1] - phi[:-2, 1:-1, 1:-1]) / (2 * dx),
            -(phi[1:-1, 2:, 1:-1] - phi[1:-1, :-2, 1:-1]) / (2 * dy),
            -(phi[1:-1, 1:-1, 2:] - phi[1:-1, 1:-1, :-2]) / (2 * dz))


def _rel(a, b):
    return np.max(np.abs(a / b - 1.0))


def test_fodo_1000_steps_plain_and_mixed_against_oracle():
    torch.cuda.set_device(0)
    g = np.load(FIXTURE)
    ex, ey, live, vc, phi_p, parts_p = _run("fp64", g)
    dev = max(_rel(ex, g["epsx"]), _rel(ey, g["epsy"]))
    nvc = int(np.sum(vc != g["vcycles"]))
    print("plain: max rel emittance deviation %.2e over %d periods; V-cycles %d (oracle %d), %d solves differ" % (
        dev, len(ex), vc.sum(), g["vcycles"].sum(), nvc))
    assert np.array_equal(live, g["live"])
    assert dev <= 1e-9
    assert nvc <= 2
    ex, ey, live, vc, phi_m, parts_m = _run("mixed", g)
    dev = max(_rel(ex, g["epsx"]), _rel(ey, g["epsy"]))
    dphi = np.max(np.abs(phi_m - phi_p)) / np.max(np.abs(phi_p))
    dE = max(np.max(np.abs(a - b)) / np.max(np.abs(b)) for a, b in zip(_efield(phi_m), _efield(phi_p)))
    both = (parts_p["gaminv"] != 0) & (parts_m["gaminv"] != 0)
    dps = {k: np.sqrt(np.mean((parts_m[k][both] - parts_p[k][both]) ** 2)) / np.std(parts_p[k][both])
           for k in ("x", "y", "ux", "uy")}
    print("mixed after 1000 steps: phi within %.2e and E within %.2e of max|.| of the FP64 run" % (dphi, dE))
    print("mixed after 1000 steps: rms phase-space difference / rms value: %s" %
          " ".join("%s %.2e" % kv for kv in dps.items()))
    print("mixed: max rel emittance deviation %.2e; after 1000 steps x %.2e y %.2e; V-cycles %d; live %d vs %d" % (
        dev, abs(ex[-1] / g["epsx"][-1] - 1), abs(ey[-1] / g["epsy"][-1] - 1), vc.sum(), live[-1], g["live"][-1]))
    assert np.max(np.abs(live - g["live"])) <= 2
    assert dev <= 1e-4
    assert dphi <= 1e-4 and dE <= 1e-4
    assert max(dps.values()) <= 1e-4
