"""GPU multigrid parity: the reference's known-answer test on the B200
(every boundary combination, error < 1e-10 at mgtol 1e-12) and bit-for-bit
agreement with the FP64 oracle given the same rho, phi and conductors."""
import numpy as np
import pytest

from oracle import oracle
from tests import gpu_helpers as H
from tests import mgkat

pytestmark = pytest.mark.gpu

COMBOS = mgkat.boundary_combos()


@pytest.mark.parametrize("bounds", COMBOS, ids=["".join(map(str, b)) for b in COMBOS])
def test_gpu_mg_kat_bitexact(bounds):
    dx, dy, dz, *_ = mgkat.mesh()
    rho, phi0, expected = mgkat.setup(bounds, oracle.eps0())
    s = H.make_solver(mgkat.NX, mgkat.NY, mgkat.NZ, (-1, -1, -1), (1, 1, 1), bounds, mgtol=1e-12)
    s.rho = rho
    s.phi = phi0
    s.solve()
    gphi = s.phi.cpu().numpy()
    ophi = phi0.copy(order="F")
    it, err = oracle.mgsolve(ophi, rho, dx, dy, dz, bounds, mgtol=1e-12)
    assert s.mgiters == it
    assert s.mgiters < 100
    assert mgkat.error(gphi, expected, bounds) < 1e-10
    assert np.array_equal(gphi, ophi), "max |gpu - oracle| = %g" % np.max(np.abs(gphi - ophi))


def _conductor_case(nx=32, ny=32, nz=48):
    from warp_b200 import conductors as C
    mins, maxs = (-0.5, -0.5, -0.5), (0.5, 0.5, 0.5)
    shapes = [C.ZCylinderOut(radius=0.45, length=10.0, voltage=0.0),
              C.Sphere(radius=0.12, voltage=0.7, xcent=0.15, ycent=-0.1, zcent=0.1),
              C.Sphere(radius=0.09, voltage=-0.4, xcent=-0.2, ycent=0.12, zcent=-0.2),
              C.ZCylinder(radius=0.05, length=0.5, voltage=0.3, xcent=-0.1, ycent=-0.2, zcent=0.1)]
    s = H.make_solver(nx, ny, nz, mins, maxs, (0, 0, 0, 0, 0, 0), mgtol=1e-10)
    for sh in shapes:
        s.installconductor(sh)
    rho = H.gaussian_blobs_rho(nx, ny, nz, mins, maxs, 8, 1, oracle.eps0())
    return s, shapes, rho


def test_gpu_conductor_data_matches_oracle():
    s, shapes, _ = _conductor_case()
    s.getconductorobject()
    mine = H.as_set(s.conductor_data())
    oc = H.oracle_conductors(s, shapes)
    ref = H.as_set(oc.export())
    assert len(mine[0]) > 0 and len(mine[1]) > 0
    assert mine[0] == ref[0]
    assert mine[1] == ref[1]


# nz = 47: an odd periodic z, where the nodes (i, j, 0) and (i, j, nz-1) have
# the same colour and the periodic images must keep their values through a
# half pass
@pytest.mark.parametrize("bounds,nz", [((0, 0, 0, 0, 0, 0), 48), ((0, 0, 0, 0, 2, 2), 48), ((1, 1, 0, 0, 2, 2), 48),
                                       ((0, 0, 0, 0, 2, 2), 47), ((0, 0, 0, 0, 0, 0), 47)])
def test_gpu_mg_conductors_bitexact(bounds, nz):
    s, shapes, rho = _conductor_case(nz=nz)
    s.bounds = list(bounds)
    # bounds are fixed at construction; rebuild with the wanted ones
    s2 = H.make_solver(s.nx, s.ny, s.nz, (s.xmmin, s.ymmin, s.zmmin), (s.xmmax, s.ymmax, s.zmmax), bounds,
                       mgtol=1e-10)
    for sh in shapes:
        s2.installconductor(sh)
    s2.rho = rho
    s2.phi = np.zeros((s2.nx + 3, s2.ny + 3, s2.nz + 3), order="F")
    s2.solve()
    gphi = s2.phi.cpu().numpy()
    oc = H.oracle_conductors(s2, shapes)
    ophi = np.zeros_like(gphi, order="F")
    it, err = oracle.mgsolve(ophi, rho, s2.dx, s2.dy, s2.dz, bounds, conductors=oc, mgtol=1e-10)
    assert s2.mgiters == it < 100
    assert np.array_equal(gphi, ophi), "max |gpu - oracle| = %g" % np.max(np.abs(gphi - ophi))
    # conductor potentials hold exactly on interior points of the finest level
    ii, iv, il = oc.export()["interior"]
    sel = il == 0
    idx = ii[sel] + 1
    assert np.array_equal(gphi[idx[:, 0], idx[:, 1], idx[:, 2]], iv[sel])


# MultiGrid3D's solver options away from their defaults: over-relaxation,
# several or no down passes, extra up passes, fewer levels, and the
# conductor stencil without the subgrid distances (lcndbndy False)
OPTIONS = [dict(mgparam=1.5), dict(downpasses=2, uppasses=3), dict(downpasses=0, uppasses=2),
           dict(mgmaxlevels=3), dict(mgparam=1.0, downpasses=1, uppasses=2, mgmaxlevels=4),
           dict(lcndbndy=False, mgtol=1e-6)]


@pytest.mark.parametrize("opts", OPTIONS, ids=["-".join("%s%s" % kv for kv in o.items()) for o in OPTIONS])
@pytest.mark.parametrize("bounds", [(0, 0, 0, 0, 2, 2), (0, 0, 0, 0, 0, 0)])
def test_gpu_mg_solver_options_bitexact(opts, bounds):
    s, shapes, rho = _conductor_case()
    opts = dict(opts)
    mgtol = opts.pop("mgtol", 1e-9)
    sv = H.make_solver(s.nx, s.ny, s.nz, (s.xmmin, s.ymmin, s.zmmin), (s.xmmax, s.ymmax, s.zmmax), bounds,
                       mgtol=mgtol, **opts)
    for sh in shapes:
        sv.installconductor(sh)
    sv.rho = rho
    sv.phi = np.zeros((sv.nx + 3, sv.ny + 3, sv.nz + 3), order="F")
    sv.solve()
    gphi = sv.phi.cpu().numpy()
    oc = H.oracle_conductors(sv, shapes)
    ophi = np.zeros_like(gphi, order="F")
    it, err = oracle.mgsolve(ophi, rho, sv.dx, sv.dy, sv.dz, bounds, conductors=oc, mgtol=mgtol, **opts)
    assert sv.mgiters == it < 100
    assert np.array_equal(gphi, ophi), "max |gpu - oracle| = %g" % np.max(np.abs(gphi - ophi))


def test_gpu_mixed_precision_reaches_fp64_tolerance():
    s, shapes, rho = _conductor_case(64, 64, 96)
    ref = H.make_solver(s.nx, s.ny, s.nz, (s.xmmin, s.ymmin, s.zmmin), (s.xmmax, s.ymmax, s.zmmax),
                        (0, 0, 0, 0, 0, 0), mgtol=1e-12, tolkind="relres")
    mix = H.make_solver(s.nx, s.ny, s.nz, (s.xmmin, s.ymmin, s.zmmin), (s.xmmax, s.ymmax, s.zmmax),
                        (0, 0, 0, 0, 0, 0), mgtol=1e-10, tolkind="relres", precision="mixed")
    for sv in (ref, mix):
        for sh in shapes:
            sv.installconductor(sh)
        sv.rho = rho
        sv.solve()
        assert sv.converged
    assert mix.relres <= 1e-10
    assert mix.relresidual() <= 1e-10
    a, b = ref.phi.cpu().numpy(), mix.phi.cpu().numpy()
    assert np.max(np.abs(a - b)) <= 1e-8 * np.max(np.abs(a))


def test_gpu_relres_tolerance_fp64():
    s, shapes, rho = _conductor_case()
    s2 = H.make_solver(s.nx, s.ny, s.nz, (s.xmmin, s.ymmin, s.zmmin), (s.xmmax, s.ymmax, s.zmmax),
                       (0, 0, 0, 0, 0, 0), mgtol=1e-6, tolkind="relres")
    for sh in shapes:
        s2.installconductor(sh)
    s2.rho = rho
    s2.solve()
    assert s2.converged and s2.relres <= 1e-6
    oc = H.oracle_conductors(s2, shapes)
    ophi = s2.phi.cpu().numpy().copy(order="F")
    assert oracle.relresidual(ophi, rho, s2.dx, s2.dy, s2.dz, (0,) * 6, oc) == pytest.approx(s2.relres, rel=1e-9)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_gpu_graph_replay_equals_eager(precision):
    """V-cycles replayed from a captured CUDA graph give the same bits as the
    kernel-by-kernel launches."""
    s, shapes, rho = _conductor_case()
    out = []
    for graphs in (False, True):
        sv = H.make_solver(s.nx, s.ny, s.nz, (s.xmmin, s.ymmin, s.zmmin), (s.xmmax, s.ymmax, s.zmmax),
                           (0, 0, 0, 0, 2, 2), mgtol=1e-9, tolkind="relres", precision=precision,
                           use_graphs=graphs)
        for sh in shapes:
            sv.installconductor(sh)
        sv.rho = rho
        sv.solve()
        sv.solve()  # second solve replays the cached graph
        out.append((sv.phi.cpu().numpy(), sv.mgiters))
    assert out[0][1] == out[1][1]
    assert np.array_equal(out[0][0], out[1][0])


def test_gpu_field_energy_bitexact():
    """getese3dfromrhophi: the GPU sum in the reference's order equals the
    oracle bit for bit, on a solved field."""
    s, shapes, rho = _conductor_case()
    s.rho = rho
    s.solve()
    e = s.getese()
    ref = oracle.ese(rho, s.phi.cpu().numpy(), s.dx, s.dy, s.dz)
    assert e == ref
    assert e != 0.0


def test_gpu_find_mgparam_tunes_a_converging_solver():
    """MultiGrid3D.find_mgparam on the conductor problem: the parameters it
    settles on are in range and solve the problem within mgmaxiters."""
    s, shapes, rho = _conductor_case()
    for sh in shapes:
        s.installconductor(sh)
    s.rho = rho
    s.phi = np.zeros((s.nx + 3, s.ny + 3, s.nz + 3), order="F")
    s.solve()
    default_iters = s.mgiters
    s.find_mgparam(log=lambda *a: None)
    assert 0.01 < s.mgparam <= 2.0 and s.downpasses >= 1 and s.uppasses >= 1
    s.phi = np.zeros((s.nx + 3, s.ny + 3, s.nz + 3), order="F")
    s.solve()
    assert s.converged and s.mgiters < s.mgmaxiters
    print("find_mgparam: mgparam %.3f, passes %d/%d, V-cycles %d (default %d)" % (
        s.mgparam, s.downpasses, s.uppasses, s.mgiters, default_iters))


def test_gpu_setconductorvoltage_matches_oracle():
    """setconductorvoltage changes one conductor's voltage (by id or by the
    conductor object); the next solve equals the oracle's with the new
    voltage bit for bit."""
    s, shapes, rho = _conductor_case()
    for sh in shapes:
        s.installconductor(sh)
    s.rho = rho
    s.solve()
    s.setconductorvoltage(1.3, condid=shapes[1].condid)
    s.setconductorvoltage(-0.9, condid=shapes[3])
    assert shapes[1].voltage == 1.3 and shapes[3].voltage == -0.9
    s.phi = np.zeros((s.nx + 3, s.ny + 3, s.nz + 3), order="F")
    s.solve()
    gphi = s.phi.cpu().numpy()
    oc = H.oracle_conductors(s, shapes)
    ophi = np.zeros_like(gphi, order="F")
    it, err = oracle.mgsolve(ophi, rho, s.dx, s.dy, s.dz, (0,) * 6, conductors=oc, mgtol=1e-10)
    assert s.mgiters == it
    assert np.array_equal(gphi, ophi)
    with pytest.raises(NotImplementedError):
        s.setconductorvoltage([0.0] * (s.nz + 1), condid=shapes[1].condid)
