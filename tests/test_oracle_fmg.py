"""The oracle's full multigrid (fullmultigrid3dsolve, f3d_mgrid.F:502-945,
behind FullMultiGrid3D, scripts/multigrid.py:957) against the reference's
known-answer test (warp_test/MutltiGrid3D_test.py). Full multigrid sets phi
to zero before expanding the coarse solution into it, Dirichlet boundary
planes included, so it solves with grounded Dirichlet faces: of the 125
boundary combinations, the 8 without a Dirichlet face must meet the test's
1e-10 bound, and the others must not (their manufactured boundary values are
not zero). With grounded faces and conductors it must reach the same
solution as multigrid3dsolve."""
import numpy as np
import pytest

from oracle import oracle
from tests import gpu_helpers as H
from tests import mgkat

NO_DIRICHLET = [b for b in mgkat.boundary_combos() if 0 not in b]


def test_eight_combinations_have_no_dirichlet_face():
    assert len(NO_DIRICHLET) == 8


@pytest.mark.parametrize("bounds", NO_DIRICHLET, ids=["".join(map(str, b)) for b in NO_DIRICHLET])
def test_oracle_fmg_kat(bounds):
    dx, dy, dz, *_ = mgkat.mesh()
    rho, phi, expected = mgkat.setup(bounds, oracle.eps0())
    iters, err = oracle.mgsolve(phi, rho, dx, dy, dz, bounds, mgtol=1e-12, mgmaxvcycles=2)
    assert iters < 100
    assert mgkat.error(phi, expected, bounds) < 1e-10


def test_oracle_fmg_drops_nonzero_dirichlet_values():
    bounds = (0, 0, 0, 0, 0, 0)
    dx, dy, dz, *_ = mgkat.mesh()
    rho, phi, expected = mgkat.setup(bounds, oracle.eps0())
    oracle.mgsolve(phi, rho, dx, dy, dz, bounds, mgtol=1e-12, mgmaxvcycles=2)
    assert np.abs(phi[1, 1:-1, 1:-1]).max() == 0.0
    assert mgkat.error(phi, expected, bounds) > 1e-3


@pytest.mark.parametrize("bounds", [(0, 0, 0, 0, 2, 2), (1, 0, 0, 1, 0, 0)])
def test_oracle_fmg_matches_multigrid_with_conductors(bounds):
    nx, ny, nz = 32, 32, 48
    mins, maxs = (-0.04, -0.04, 0.0), (0.04, 0.04, 0.6)
    dx, dy, dz = 0.08 / nx, 0.08 / ny, 0.6 / nz
    rho = H.gaussian_blobs_rho(nx, ny, nz, mins, maxs, 5, 7, oracle.eps0())
    oc = oracle.Conductors(nx, ny, nz, dx, dy, dz, *mins)
    oc.add_shape("ZCylinderOut", 0.035, 100.0, 0.0, 0.0, 0.0, 0.3)
    oc.add_shape("Sphere", 0.008, 0.0, 5.0, 0.01, 0.0, 0.3, condid=2)
    oc.finalize()
    a = np.zeros((nx + 3, ny + 3, nz + 3), order="F")
    b = np.zeros_like(a, order="F")
    oracle.mgsolve(a, rho, dx, dy, dz, bounds, conductors=oc, mgtol=1e-11)
    it, err = oracle.mgsolve(b, rho, dx, dy, dz, bounds, conductors=oc, mgtol=1e-11, mgmaxvcycles=2)
    assert it < 100
    assert np.abs(a - b).max() <= 1e-9 * np.abs(a).max()
