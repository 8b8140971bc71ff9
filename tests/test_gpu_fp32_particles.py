"""FP32 particle storage, the particle arrays of the mixed-precision form
(wg_particles_f32 and the _f32 entry points), against the FP64 path and the
oracle.

- Deposit: the FP32 positions are widened to FP64 before the fixed-point
  weights are formed, so rho equals the FP64 deposit of the rounded
  positions bit for bit, and the oracle's FP64 running sum within 1e-13.
- Advance: E is gathered in FP64 at the FP32 positions, the kicks, rotation
  and drift run in FP32. After a halfv, two fullv and a synchv step with
  quads and the pipe (in a random phi of 1 kV rms, which makes the kicks
  large), positions agree with the oracle's FP64 push of the same starting
  values within 1e-6 and velocities within 1e-5 of each component's
  largest magnitude (measured on the B200: 1.6e-7 and 2.1e-6).
- Sort keys, the permutation and the moments see the same numbers as the
  FP64 path on the widened arrays."""
import numpy as np
import pytest
import torch

from oracle import oracle
from tests import gpu_helpers as H

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "z", "ux", "uy", "uz", "gaminv")


def _setup(npart=200_000, seed=3):
    from warp_b200 import pic
    from warp_b200.particles import semigaussian
    cfg = pic.workload("A")
    p = semigaussian(npart, seed=seed, radius=4e-3, mismatch=0.2, angle_rms=5e-3)
    s = H.make_solver(cfg["nx"], cfg["ny"], cfg["nz"], (cfg["xmmin"], cfg["ymmin"], cfg["zmmin"]),
                      (cfg["xmmax"], cfg["ymmax"], cfg["zmmax"]), (0, 0, 0, 0, 2, 2))
    return cfg, s, p


def _rounded(p):
    """The FP32 values of p, as FP64 arrays."""
    return {k: v.astype(np.float32).astype(np.float64) for k, v in p.items()}


def _groups(p, w=1e4):
    from warp_b200.particles import ParticleGroup
    return (ParticleGroup(p, w=w, dtype=torch.float32), ParticleGroup(_rounded(p), w=w))


def test_deposit_f32_is_the_fp64_deposit_of_the_rounded_positions():
    cfg, s, p = _setup()
    p["gaminv"][::97] = 0.0
    g32, g64 = _groups(p)
    assert g32.x.dtype == torch.float32 and g32.x.element_size() == 4
    s.loadrho(pgroups=[g32])
    a = s.rho.cpu().numpy()
    s.loadrho(pgroups=[g64])
    b = s.rho.cpu().numpy()
    assert np.array_equal(a, b)
    pr = _rounded(p)
    ref = np.zeros((s.nx + 1, s.ny + 1, s.nz + 1), order="F")
    oracle.setrho(ref, pr["x"], pr["y"], pr["z"], g32.q, g32.w, s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin,
                  gaminv=pr["gaminv"])
    oracle.rhobc(ref, s.bounds)
    assert np.max(np.abs(a - ref)) <= 1e-13 * np.max(np.abs(ref))
    # chunked form
    s.deposit_begin()
    s.deposit_add(g32, 0, 70_000)
    s.deposit_add(g32, 70_000, None)
    s.deposit_end(zero_first=True)
    assert np.array_equal(s.rho.cpu().numpy(), a)


def test_advance_f32_against_the_fp64_oracle():
    from warp_b200 import pic
    from warp_b200.lattice import fodo
    from warp_b200.particles import ParticleGroup
    cfg, s, p = _setup(100_000)
    rng = np.random.default_rng(11)
    phi = np.asfortranarray(1e3 * rng.standard_normal((s.nx + 3, s.ny + 3, s.nz + 3)))
    s.phi = phi
    s.setlattice(fodo(cfg["quad_gradient"], cfg["quad_length"], cfg["period"]))
    czs, cze, cdb, nzl, zlmin, dzl = s._lattice
    dt = pic.timestep(cfg)
    p["x"][:1000] *= 8.6  # some cross the pipe
    ref = _rounded(p)
    pg = ParticleGroup(p, w=1.0, dtype=torch.float32)
    for center in ("halfv", "fullv", "fullv", "synchv"):
        ex, ey, ez = oracle.sete(phi, ref["x"], ref["y"], ref["z"], s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin)
        oracle.push(ref, ex, ey, ez, pg.q, pg.m, dt, (czs, cze, cdb), zlmin, dzl, s.zmmin, s.zmmax,
                    cfg["pipe_radius"], center=center)
        s.advance(pg, dt, prwall=cfg["pipe_radius"], center=center)
    got = {k: v.astype(np.float64) for k, v in pg.to_numpy().items()}
    lost_ref, lost = ref["gaminv"] == 0, got["gaminv"] == 0
    assert lost_ref.sum() > 0
    assert np.sum(lost_ref != lost) <= 2
    both = ~lost_ref & ~lost
    errs = {}
    for k in ("x", "y", "z", "ux", "uy", "uz"):
        errs[k] = np.max(np.abs(got[k][both] - ref[k][both])) / np.max(np.abs(ref[k][both]))
    print("FP32 push vs FP64 oracle after 4 steps (max abs error / max abs value):",
          " ".join("%s %.2e" % kv for kv in errs.items()))
    for k, e in errs.items():
        assert e <= (1e-6 if k in ("x", "y", "z") else 1e-5), (k, e)


def test_sort_and_moments_f32_see_the_fp64_numbers():
    cfg, s, p = _setup(150_000)
    p["gaminv"][::31] = 0.0
    g32, g64 = _groups(p, w=1.0)
    m32, m64 = s.moments(g32), s.moments(g64)
    assert m32 == m64
    g32.sort(s)
    g64.sort(s)
    assert g32.np == g64.np == int((p["gaminv"] != 0).sum())
    a, b = g32.to_numpy(), g64.to_numpy()
    for k in KEYS:
        assert a[k].dtype == np.float32
        assert np.array_equal(a[k].astype(np.float64), b[k]), k
    uold = (g32.ux.clone(), g32.uy.clone(), g32.uz.clone())
    z32 = s.zmoments(g32, uold, 1e-9, 0.0, 1.0, 64)
    uold64 = (g64.ux.clone(), g64.uy.clone(), g64.uz.clone())
    z64 = s.zmoments(g64, uold64, 1e-9, 0.0, 1.0, 64)
    for u, v in zip(z32, z64):
        assert np.allclose(u, v, rtol=1e-12, atol=1e-12 * np.max(np.abs(v)))


def test_f32_wrap_keeps_particles_inside_z():
    """(float)zmmax can round past zmmax: the FP32 wrap must still leave every
    particle inside [zmmin, zmmax] (in FP64 terms), where the deposit's CIC
    fractions stay in [0, 1] and no weight goes negative."""
    from warp_b200.particles import ParticleGroup
    s = H.make_solver(32, 32, 64, (-0.02, -0.02, -0.36), (0.02, 0.02, 0.36), (0, 0, 0, 0, 2, 2))
    assert float(np.float32(0.36)) > 0.36  # the rounding that the wrap has to undo
    n = 4096
    rng = np.random.default_rng(4)
    dt = 1e-9
    z = np.concatenate([0.36 - rng.uniform(0, 2e-8, n // 2), -0.36 + rng.uniform(0, 2e-8, n // 2)])
    uz = np.concatenate([rng.uniform(0, 4e1, n // 2), -rng.uniform(0, 4e1, n // 2)])
    p = {"x": rng.uniform(-1e-3, 1e-3, n), "y": rng.uniform(-1e-3, 1e-3, n), "z": z, "ux": np.zeros(n),
         "uy": np.zeros(n), "uz": uz, "gaminv": np.ones(n)}
    pg = ParticleGroup(p, w=1.0, dtype=torch.float32)
    for _ in range(20):
        s.advance(pg, dt, center="fullv")
        zz = pg.z.double().cpu().numpy()
        assert zz.min() >= -0.36 and zz.max() <= 0.36
    s.loadrho(pgroups=[pg])  # WG_EOVERFLOW on a negative weight
    assert float(s.rho.sum()) * s.dx * s.dy * s.dz == pytest.approx(n * pg.q * pg.w, rel=1e-12)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_fused_advance_deposit_equals_advance_then_deposit(dtype):
    """wg_advance_deposit: the same particles as wg_advance and the same rho,
    bit for bit, as a deposit of the advanced particles, for sorted and
    unsorted particles (shared box and direct accumulator paths)."""
    from warp_b200 import pic
    from warp_b200.lattice import fodo
    from warp_b200.particles import ParticleGroup
    cfg, s, p = _setup(300_000)
    rng = np.random.default_rng(21)
    s.phi = np.asfortranarray(10. * rng.standard_normal((s.nx + 3, s.ny + 3, s.nz + 3)))
    s.setlattice(fodo(cfg["quad_gradient"], cfg["quad_length"], cfg["period"]))
    dt = pic.timestep(cfg)
    p["x"][:500] *= 8.6  # some are lost at the pipe
    a, b = ParticleGroup(p, w=1e4, dtype=dtype), ParticleGroup(p, w=1e4, dtype=dtype)
    b.sort(s)
    a.sort(s)
    for sort_first in (True, False):
        if not sort_first:  # shuffled: boxes too large for shared memory
            perm = torch.randperm(a.np, device=a.device)
            for k in KEYS:
                setattr(a, k, getattr(a, k)[perm].contiguous())
                setattr(b, k, getattr(b, k)[perm].contiguous())
        for center in ("halfv", "fullv", "fullv"):
            s.advance(a, dt, prwall=cfg["pipe_radius"], center=center)
            s.loadrho(pgroups=[a])
            r1 = s.rho.cpu().numpy()
            s.deposit_begin()
            s.advance(b, dt, prwall=cfg["pipe_radius"], center=center, deposit=True)
            s.deposit_end(zero_first=True)
            r2 = s.rho.cpu().numpy()
            assert np.array_equal(r1, r2), (sort_first, center)
            for k in KEYS:
                assert torch.equal(getattr(a, k), getattr(b, k)), (sort_first, center, k)
    assert int((a.gaminv == 0).sum()) > 0
    # without an open deposit the fused call is refused
    import ctypes
    from warp_b200 import _lib
    prm = _lib.PushParams(dt, 1e30, 0., 0., 0, 0)
    st = b.cstruct()
    assert b.fn("wg_advance_deposit")(s._h, ctypes.byref(st), ctypes.byref(prm)) == -3
