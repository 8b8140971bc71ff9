"""Full multigrid (FullMultiGrid3D / fullmultigrid3dsolve, f3d_mgrid.F:
502-945) on the B200 against the oracle's, bit for bit: the same level-0
V-cycle count and the same phi, for every boundary combination of the
reference's known-answer test and for a grid with conductors at non-zero
voltage. The mixed-precision form starting from the full multigrid's phi
must reach its relative residual; a grid with a single level keeps its
warm start."""
import numpy as np
import pytest

from oracle import oracle
from tests import gpu_helpers as H
from tests import mgkat

pytestmark = pytest.mark.gpu

COMBOS = mgkat.boundary_combos()


def _fmg_solver(*args, **kw):
    from warp_b200.multigrid import FullMultiGridB200
    mins, maxs, bounds = args[3], args[4], args[5]
    return FullMultiGridB200(args[0], args[1], args[2], mins[0], maxs[0], mins[1], maxs[1], mins[2], maxs[2],
                             bounds=bounds, mgverbose=-1, **kw)


@pytest.mark.parametrize("bounds", COMBOS, ids=["".join(map(str, b)) for b in COMBOS])
def test_gpu_fmg_kat_bitexact(bounds):
    dx, dy, dz, *_ = mgkat.mesh()
    rho, phi0, expected = mgkat.setup(bounds, oracle.eps0())
    s = _fmg_solver(mgkat.NX, mgkat.NY, mgkat.NZ, (-1, -1, -1), (1, 1, 1), bounds, mgtol=1e-12)
    s.rho = rho
    s.phi = phi0
    s.solve()
    gphi = s.phi.cpu().numpy()
    ophi = phi0.copy(order="F")
    it, err = oracle.mgsolve(ophi, rho, dx, dy, dz, bounds, mgtol=1e-12, mgmaxvcycles=2)
    assert s.mgiters == it < 100
    assert np.array_equal(gphi, ophi), "max |gpu - oracle| = %g" % np.max(np.abs(gphi - ophi))
    if 0 not in bounds:
        assert mgkat.error(gphi, expected, bounds) < 1e-10


@pytest.mark.parametrize("mgmaxvcycles", [1, 2, 3])
def test_gpu_fmg_conductors_bitexact(mgmaxvcycles):
    from warp_b200 import conductors as C
    nx, ny, nz = 32, 32, 64
    mins, maxs = (-0.04, -0.04, 0.0), (0.04, 0.04, 1.0)
    bounds = (0, 0, 0, 0, 2, 2)
    shapes = [C.ZCylinderOut(radius=0.035, length=100.0, zcent=0.5),
              C.ZCylinder(radius=0.008, length=100.0, voltage=50.0, xcent=0.015, zcent=0.5)]
    s = _fmg_solver(nx, ny, nz, mins, maxs, bounds, mgtol=1e-9, mgmaxvcycles=mgmaxvcycles)
    for sh in shapes:
        s.installconductor(sh)
    rho = H.gaussian_blobs_rho(nx, ny, nz, mins, maxs, 6, 3, oracle.eps0())
    s.rho = rho
    s.phi = np.ones((nx + 3, ny + 3, nz + 3), order="F")  # not used by the full multigrid
    s.solve()
    oc = H.oracle_conductors(s, shapes)
    ophi = np.zeros((nx + 3, ny + 3, nz + 3), order="F")
    it, err = oracle.mgsolve(ophi, rho, s.dx, s.dy, s.dz, bounds, conductors=oc, mgtol=1e-9,
                             mgmaxvcycles=mgmaxvcycles)
    assert s.mgiters == it < 100
    gphi = s.phi.cpu().numpy()
    assert np.array_equal(gphi, ophi), "max |gpu - oracle| = %g" % np.max(np.abs(gphi - ophi))


def test_gpu_fmg_mixed_precision_reaches_relres():
    from warp_b200 import conductors as C
    nx, ny, nz = 64, 64, 128
    mins, maxs = (-0.04, -0.04, 0.0), (0.04, 0.04, 1.0)
    rho = H.gaussian_blobs_rho(nx, ny, nz, mins, maxs, 6, 4, oracle.eps0())
    out = {}
    for prec in ("fp64", "mixed"):
        s = _fmg_solver(nx, ny, nz, mins, maxs, (0, 0, 0, 0, 2, 2), tolkind="relres", mgtol=1e-10,
                        precision=prec)
        s.installconductor(C.ZCylinderOut(radius=0.035, length=100.0, zcent=0.5))
        s.rho = rho
        s.solve()
        assert s.converged and s.relres <= 1e-10
        out[prec] = s.phi.cpu().numpy()
    assert np.abs(out["fp64"] - out["mixed"]).max() <= 1e-8 * np.abs(out["fp64"]).max()


def test_gpu_fmg_single_level_keeps_warm_start():
    bounds = (1, 1, 0, 0, 2, 2)
    s = _fmg_solver(2, 2, 2, (0., 0., 0.), (1., 1., 1.), bounds, mgtol=1e-12)
    rng = np.random.default_rng(5)
    rho = np.asfortranarray(rng.standard_normal((3, 3, 3))) * 1e-9
    phi0 = np.asfortranarray(rng.standard_normal((5, 5, 5)))
    s.rho = rho
    s.phi = phi0
    s.solve()
    ref = phi0.copy(order="F")
    it, err = oracle.mgsolve(ref, rho, 0.5, 0.5, 0.5, bounds, mgtol=1e-12, mgmaxvcycles=2)
    assert s.mgiters == it
    assert np.array_equal(s.phi.cpu().numpy(), ref)
