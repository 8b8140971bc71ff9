"""The reference's integration test, warp_test/basicFODO_test.py, rebuilt:
a matched 80 keV K+ beam (2 mA, 62.47 mm mrad) in a FODO lattice of
hard-edge quads (11 cm long, +-8.4818 T/m, half period 36 cm; sigma0 = 72
and sigma = 20 degrees). The PIC rms envelope, twice the rms size on the z
grid, must follow the KV envelope:
- within 0.5 mm after loading;
- within 1 mm after one lattice period of 50 steps.
These are the test's own tolerances. Differences from the reference test:
- the full transverse domain 32 x 32 replaces the quarter domain 16 x 16
  with four-fold symmetry;
- 2e5 pseudo-random particles replace 2e4 digit-reversed ones, to keep the
  per-slice rms noise below 0.2 mm;
- the envelope comes from warp_b200.envelope instead of the env package.
Everything else runs through the GPU PIC step: deposit, multigrid, gather,
quads and Boris push.
"""
import numpy as np
import pytest
import torch

from tests.fodo_setup import A0, B0, EMIT, HLP, IBEAM, PIPERAD
from tests.fodo_setup import lattice as _lattice
from tests.fodo_setup import species as _species

pytestmark = pytest.mark.gpu


def test_basic_fodo_rms_envelope_follows_kv_envelope():
    from warp_b200.envelope import integrate
    from warp_b200.multigrid import MultiGridB200
    from warp_b200.particles import ParticleGroup, rms_along_z, semigaussian_matched
    torch.cuda.set_device(0)
    q, m, v, gamma = _species()
    lat = _lattice()
    z, a, b, ap, bp = integrate(lat, q, m, v, IBEAM, EMIT, EMIT, A0, B0, 0., 0., z0=-HLP, gamma=gamma)
    nx, ny, nz, npart = 32, 32, 64, 200_000
    s = MultiGridB200(nx, ny, nz, -PIPERAD, PIPERAD, -PIPERAD, PIPERAD, -HLP, HLP, bounds=(0, 0, 0, 0, 2, 2),
                      tolkind="relres", mgtol=1e-8)
    s.setlattice(lat)
    gen = torch.Generator(device="cuda").manual_seed(72)
    beam = semigaussian_matched(npart, gen, z, a, b, ap, bp, EMIT, EMIT, -HLP, HLP, v)
    w = IBEAM * (2 * HLP) / (q * v * npart)
    pg = ParticleGroup(beam, q=q, m=m, w=w)
    s.addpgroup(pg)
    zn = -HLP + np.arange(nz + 1) * (2 * HLP / nz)
    aenv, benv = np.interp(zn, z, a), np.interp(zn, z, b)
    xr, yr = rms_along_z(pg, -HLP, HLP, nz)
    d0 = max(np.abs(2 * xr - aenv).max(), np.abs(2 * yr - benv).max())
    s.loadrho()
    s.solve()
    dt = (2 * HLP / 50) / v
    for it in range(50):
        # the loaded velocities are at t = 0: the first step is halfv
        s.advance(pg, dt, prwall=PIPERAD, center="halfv" if it == 0 else "fullv")
        s.loadrho()
        s.solve()
        assert s.converged
    xr, yr = rms_along_z(pg, -HLP, HLP, nz)
    d1x, d1y = np.abs(2 * xr - aenv).max(), np.abs(2 * yr - benv).max()
    print("FODO: envelope a %.2f-%.2f mm; max |2 rms - env|: load %.3f mm, one period x %.3f mm, y %.3f mm; "
          "live %d" % (1e3 * a.min(), 1e3 * a.max(), 1e3 * d0, 1e3 * d1x, 1e3 * d1y, pg.nlive()))
    assert d0 <= 0.0005
    assert d1x <= 0.001 and d1y <= 0.001
    assert pg.nlive() >= 0.999 * npart
