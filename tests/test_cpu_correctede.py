"""The oracle's lcorrectede gather (sete3dwithconductor with efetch = 1,
f3d_mgrid.F:4774-5220, and the field at the subgrid points,
getefieldatconductorsubgrid, :4635-4735) on a coaxial line: a rod at 1 kV of
radius r0 inside a grounded pipe of radius R, where E_r = V / (r ln(R/r0)).
Next to the rod the corrected field must be several times closer to that
than the plain centred-difference gather; away from conductors the two
gathers must agree to rounding."""
import numpy as np
import pytest

from oracle import oracle

NX = NY = 32
NZ = 8
XMIN, XMAX, ZLEN = -0.04, 0.04, 0.08
R, R0, V = 0.035, 0.011, 1000.0


@pytest.fixture(scope="module")
def coax():
    dx = (XMAX - XMIN) / NX
    dz = ZLEN / NZ
    oc = oracle.Conductors(NX, NY, NZ, dx, dx, dz, XMIN, XMIN, 0.0)
    oc.add_shape("ZCylinderOut", R, 10.0, 0.0, 0.0, 0.0, ZLEN / 2)
    oc.add_shape("ZCylinder", R0, 10.0, V, 0.0, 0.0, ZLEN / 2, condid=2)
    oc.finalize()
    phi = np.zeros((NX + 3, NY + 3, NZ + 3), order="F")
    rho = np.zeros((NX + 1, NY + 1, NZ + 1), order="F")
    oracle.mgsolve(phi, rho, dx, dx, dz, (0, 0, 0, 0, 2, 2), conductors=oc, mgtol=1e-12)
    return oc, phi, dx, dz


def test_corrected_field_is_closer_to_the_coaxial_field(coax):
    oc, phi, dx, dz = coax
    rng = np.random.default_rng(0)
    n = 4000
    r = rng.uniform(R0, 0.03, n)
    th = rng.uniform(0, 2 * np.pi, n)
    x, y, z = r * np.cos(th), r * np.sin(th), rng.uniform(0, ZLEN, n)
    er = V / (r * np.log(R / R0))
    plain = oracle.sete(phi, x, y, z, dx, dx, dz, XMIN, XMIN, 0.0)
    corr = oracle.sete_cond(oc, phi, x, y, z, dx, dx, dz, XMIN, XMIN, 0.0)
    near = r < R0 + 1.5 * dx

    def rel(e):
        return np.hypot(e[0] - er * np.cos(th), e[1] - er * np.sin(th)) / er

    ep, ec = rel(plain), rel(corr)
    rms = lambda a: float(np.sqrt(np.mean(a * a)))
    assert rms(ec[near]) < 0.05 and rms(ep[near]) > 4 * rms(ec[near])
    # far from both conductors the cells are all vacuum: same field
    far = (r > R0 + 3 * dx) & (r < R - 3 * dx)
    for a, b in zip(plain, corr):
        assert np.allclose(a[far], b[far], rtol=1e-12, atol=1e-9)


def test_particles_outside_the_grid_get_no_field(coax):
    oc, phi, dx, dz = coax
    x = np.array([XMIN - 1e-3, 0.0, 0.0, XMAX + 1e-6])
    y = np.array([0.0, XMAX + 1e-3, 0.02, 0.0])
    z = np.array([0.01, 0.01, -1e-3, 0.01])
    ex, ey, ez = oracle.sete_cond(oc, phi, x, y, z, dx, dx, dz, XMIN, XMIN, 0.0)
    assert not ex.any() and not ey.any() and not ez.any()
