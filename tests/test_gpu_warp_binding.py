"""The WARP-side binding (warp_b200/warp_binding.py) driven the way WARP's
step drives a registered MultiGrid3D, on stand-ins of WARP's objects
(tests/warp_standins.py): WARP conductor objects installed through
installconductor; loadrho's zeroing, per-batch setsourcepatposition and rho
boundary conditions; dosolve with WARP's guarded potential as warm start;
fetchfieldfrompositions into WARP's E arrays. Against the oracle on the same
inputs: rho within the fixed-point rounding, the potential (guard cells
included) and V-cycle count bit for bit, E bit for bit."""
import numpy as np
import pytest
import torch

from oracle import oracle
from tests import warp_standins as W

pytestmark = pytest.mark.gpu


def _beam(n, seed):
    rng = np.random.default_rng(seed)
    r, th = 0.2 * np.sqrt(rng.random(n)), 2 * np.pi * rng.random(n)
    return {"x": r * np.cos(th), "y": r * np.sin(th), "z": rng.uniform(-0.5, 0.5, n), "ux": np.zeros(n),
            "uy": np.zeros(n), "uz": np.full(n, 1e6), "gaminv": np.ones(n)}


def test_warp_multigrid3d_binding_against_oracle():
    from warp_b200.warp_binding import gpu_multigrid, shape_from_warp
    torch.cuda.set_device(0)
    MG = gpu_multigrid(W.MultiGrid3D, W.top, W.w3d, W.f3d)
    s = MG(mgtol=1e-9)
    conds = [W.ZCylinderOut(radius=0.45, zlower=-5.0, zupper=5.0),
             W.Sphere(radius=0.12, voltage=0.7, xcent=0.15, ycent=-0.1, zcent=0.1),
             W.ZCylinder(radius=0.05, length=0.5, voltage=0.3, xcent=-0.1, ycent=-0.2, zcent=0.1)]
    for c in conds:
        s.installconductor(c)
    assert [c[0] for c in s.conductordatalist] == conds  # WARP's own list keeps WARP's objects
    q, w = 1.602e-19, 5e6
    b1, b2 = _beam(60_000, 1), _beam(40_000, 2)
    oc = oracle.Conductors(s.nx, s.ny, s.nz, s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin)
    for c in conds:
        sh = shape_from_warp(c)
        oc.add_shape({0: "ZCylinderOut", 1: "ZCylinder", 2: "Sphere"}[sh.kind], sh.radius, sh.length, sh.voltage,
                     sh.xcent, sh.ycent, sh.zcent, sh.condid)
    oc.finalize()
    phi_ref = np.zeros_like(s.potential)
    for step in range(2):
        # WARP's loadrho: zero sourcep, deposit each batch, boundary conditions
        s.sourcep[...] = 0.
        for b in (b1, b2):
            s.setsourcepatposition(b["x"], b["y"], b["z"], b["ux"], b["uy"], b["uz"], b["gaminv"], None, 0., q, w,
                                   np.array([1, 1, 1]))
        oracle.rhobc(s.source, tuple(int(v) for v in s.bounds))
        ref = np.zeros_like(s.source)
        for b in (b1, b2):
            oracle.setrho(ref, b["x"], b["y"], b["z"], q, w, s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin)
        oracle.rhobc(ref, tuple(int(v) for v in s.bounds))
        assert np.max(np.abs(s.source - ref)) <= 1e-13 * np.max(np.abs(ref))
        # dosolve(iwhich, zfact, isourcepndtscopies, indts, iselfb) from the warm start in WARP's potential
        s.dosolve(0, 1., 0, 0)
        rho = np.asfortranarray(s.source.copy())
        it, _ = oracle.mgsolve(phi_ref, rho, s.dx, s.dy, s.dz, tuple(int(v) for v in s.bounds), conductors=oc,
                               mgtol=1e-9)
        assert s.mgiters == it, (step, s.mgiters, it)
        assert np.array_equal(s.potential, phi_ref), step
        b1["z"] = (b1["z"] + 0.01 + 0.5) % 1.0 - 0.5  # the next step's particles
    # fetchfieldfrompositions adds E to WARP's arrays
    n = len(b2["x"])
    ex, ey, ez = np.ones(n), np.zeros(n), np.zeros(n)
    s.fetchfieldfrompositions(b2["x"], b2["y"], b2["z"], ex, ey, ez, None, None, None, 0)
    rx, ry, rz = oracle.sete(s.potential, b2["x"], b2["y"], b2["z"], s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin)
    assert np.array_equal(ex, 1. + rx) and np.array_equal(ey, ry) and np.array_equal(ez, rz)
    assert np.array_equal(s.getphi(), s.potential[1:-1, 1:-1, 1:-1])


def test_warp_binding_refusals():
    from warp_b200.warp_binding import gpu_multigrid
    torch.cuda.set_device(0)
    MG = gpu_multigrid(W.MultiGrid3D, W.top, W.w3d, W.f3d)
    s = MG()
    with pytest.raises(NotImplementedError):
        s.installconductor(W.Box(0.1, 0.1, 0.1))
    with pytest.raises(NotImplementedError):
        s.installconductor(W.Sphere(radius=0.1), zmin=0.)
    b = _beam(10, 3)
    with pytest.raises(NotImplementedError):
        s.setsourcepatposition(b["x"], b["y"], b["z"], b["ux"], b["uy"], b["uz"], b["gaminv"], None, 0.1, 1., 1.,
                               None)

    class T2(W.top):
        efetch = np.array([3])
    s2 = gpu_multigrid(W.MultiGrid3D, T2, W.w3d, W.f3d)()
    with pytest.raises(NotImplementedError, match="efetch"):
        s2.fetchfieldfrompositions(b["x"], b["y"], b["z"], np.zeros(10), np.zeros(10), np.zeros(10), None, None,
                                   None, 0)
