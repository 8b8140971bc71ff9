"""The KV envelope integrator against the numbers of the reference's
integration test (warp_test/basicFODO_test.py). Its FODO lattice has
sigma0 = 72 degrees, and its matched 2 mA K+ beam (a0 = 15.60 mm,
b0 = 8.76 mm, a' = b' = 0 at the focusing quad centre) has sigma = 20
degrees. The test asserts env.sig0x = 72 and env.sigx = 20."""
import math

import numpy as np
import pytest


def _setup():
    from warp_b200.constants import amu, clight, echarge
    from warp_b200.lattice import Lattice, Quad
    hlp, ql, g = 0.36, 0.11, 8.4817662372660610
    lat = Lattice([Quad(-ql / 2, ql / 2, -g), Quad(hlp - ql / 2, hlp + ql / 2, +g)], zlatperi=2 * hlp)
    m = 39.0983 * amu
    gamma = 1. + 80e3 * echarge / (m * clight * clight)
    v = math.sqrt(1. - 1. / gamma ** 2) * clight
    return lat, echarge, m, v, gamma, hlp


def test_undepressed_phase_advance_is_72_degrees():
    from warp_b200.envelope import undepressed_phase_advance
    lat, q, m, v, gamma, hlp = _setup()
    assert undepressed_phase_advance(lat, q, m, v, gamma, z0=-hlp) == pytest.approx(72.0, abs=0.1)


def test_matched_envelope_is_periodic_with_20_degree_depressed_tune():
    from warp_b200.envelope import depressed_phase_advance, integrate
    lat, q, m, v, gamma, hlp = _setup()
    emit = 62.46985327098694e-06
    z, a, b, ap, bp = integrate(lat, q, m, v, 2e-3, emit, emit, 15.60152892731585e-3, 8.75924684128793e-3,
                                z0=-hlp, gamma=gamma)
    assert abs(a[-1] - a[0]) <= 2e-5 and abs(b[-1] - b[0]) <= 2e-5
    assert abs(ap[-1]) <= 5e-5 and abs(bp[-1]) <= 5e-5
    assert depressed_phase_advance(z, a, emit) == pytest.approx(20.0, abs=0.1)
    assert depressed_phase_advance(z, b, emit) == pytest.approx(20.0, abs=0.1)
    # the quads swap the roles of a and b half a period later
    mid = np.argmin(np.abs(z))
    assert a[mid] == pytest.approx(b[0], rel=2e-3) and b[mid] == pytest.approx(a[0], rel=2e-3)


def test_envelope_without_space_charge_or_emittance_is_a_drift():
    from warp_b200.envelope import integrate
    from warp_b200.lattice import Lattice, Quad
    lat = Lattice([Quad(0.0, 0.1, 0.0)], zlatperi=1.0)
    z, a, b, ap, bp = integrate(lat, 1.6e-19, 1e-25, 1e6, 0.0, 0.0, 0.0, 1e-3, 2e-3, 1e-3, -1e-3, z0=0.0)
    assert np.allclose(a, 1e-3 + 1e-3 * (z - z[0]), rtol=0, atol=1e-12)
    assert np.allclose(b, 2e-3 - 1e-3 * (z - z[0]), rtol=0, atol=1e-12)
