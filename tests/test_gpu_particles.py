"""GPU particle kernels against the oracle: fixed-point CIC deposition
(within the fixed-point rounding, bit-identical under any particle order),
the field gather and the fused advance in its fullv, halfv and synchv forms
(bit for bit), and moments."""
import numpy as np
import pytest
import torch

from oracle import oracle
from tests import gpu_helpers as H

pytestmark = pytest.mark.gpu


def _setup(npart=200_000, seed=3):
    from warp_b200 import pic
    from warp_b200.particles import ParticleGroup, semigaussian
    cfg = pic.workload("A")
    p = semigaussian(npart, seed=seed, radius=4e-3, mismatch=0.2, angle_rms=5e-3)
    s = H.make_solver(cfg["nx"], cfg["ny"], cfg["nz"], (cfg["xmmin"], cfg["ymmin"], cfg["zmmin"]),
                      (cfg["xmmax"], cfg["ymmax"], cfg["zmmax"]), (0, 0, 0, 0, 2, 2))
    pg = ParticleGroup(p, w=1e4)
    return cfg, s, p, pg


def _oracle_rho(s, p, w, q):
    rho = np.zeros((s.nx + 1, s.ny + 1, s.nz + 1), order="F")
    oracle.setrho(rho, p["x"], p["y"], p["z"], q, w, s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin,
                  gaminv=p["gaminv"])
    oracle.rhobc(rho, s.bounds)
    return rho


def test_deposit_matches_oracle_and_is_order_independent():
    cfg, s, p, pg = _setup()
    p["gaminv"][::97] = 0.0  # some lost particles
    pg.gaminv.copy_(torch.as_tensor(p["gaminv"]))
    s.loadrho(pgroups=[pg])
    g1 = s.rho.cpu().numpy()
    ref = _oracle_rho(s, p, pg.w, pg.q)
    scale = np.max(np.abs(ref))
    assert scale > 0
    assert np.max(np.abs(g1 - ref)) <= 1e-13 * scale
    assert g1.sum() == pytest.approx(ref.sum(), rel=1e-13)
    # any particle order gives the same bits
    perm = np.random.default_rng(7).permutation(len(p["x"]))
    from warp_b200.particles import ParticleGroup
    pg2 = ParticleGroup({k: v[perm] for k, v in p.items()}, w=pg.w)
    s.loadrho(pgroups=[pg2])
    g2 = s.rho.cpu().numpy()
    assert np.array_equal(g1, g2)


def test_deposit_sorted_runs_and_lzero():
    cfg, s, p, pg = _setup(50_000)
    order = np.lexsort((p["x"], p["y"], p["z"]))
    from warp_b200.particles import ParticleGroup
    pgs = ParticleGroup({k: v[order] for k, v in p.items()}, w=pg.w)
    s.loadrho(pgroups=[pgs])
    a = s.rho.cpu().numpy()
    s.loadrho(pgroups=[pg])
    b = s.rho.cpu().numpy()
    assert np.array_equal(a, b)
    # two groups accumulate (lzero only clears before the first)
    s.loadrho(pgroups=[pg, pgs])
    c = s.rho.cpu().numpy()
    assert np.max(np.abs(c - 2 * a)) <= 1e-14 * np.max(np.abs(a)) * 4


def test_fetch_e_bitexact():
    cfg, s, p, pg = _setup(100_000)
    rng = np.random.default_rng(5)
    phi = np.asfortranarray(rng.standard_normal((s.nx + 3, s.ny + 3, s.nz + 3)))
    s.phi = phi
    s.fetche(pg)
    ex, ey, ez = oracle.sete(phi, p["x"], p["y"], p["z"], s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin)
    assert np.array_equal(pg.ex.cpu().numpy(), ex)
    assert np.array_equal(pg.ey.cpu().numpy(), ey)
    assert np.array_equal(pg.ez.cpu().numpy(), ez)
    # host-array form of the same gather
    eh = s.fetche_host(p["x"], p["y"], p["z"])
    assert np.array_equal(eh[0], ex) and np.array_equal(eh[1], ey) and np.array_equal(eh[2], ez)


def test_fetche_slice_as_warp_hands_it_over():
    """fetche(pgroup, ipmin, np) gathers particles ipmin .. ipmin+np-1
    (1-based, w3d.ipminfsapi / npfsapi) into that slice of ex/ey/ez and
    leaves the rest of the arrays alone."""
    cfg, s, p, pg = _setup(20_000)
    rng = np.random.default_rng(21)
    s.phi = np.asfortranarray(rng.standard_normal((s.nx + 3, s.ny + 3, s.nz + 3)))
    s.fetche(pg)
    whole = [pg.ex.clone(), pg.ey.clone(), pg.ez.clone()]
    for e in (pg.ex, pg.ey, pg.ez):
        e.fill_(7.0)
    s.fetche(pg, ipmin=1001, np=5000)
    for e, w in zip((pg.ex, pg.ey, pg.ez), whole):
        assert torch.equal(e[1000:6000], w[1000:6000])
        assert bool((e[:1000] == 7.0).all()) and bool((e[6000:] == 7.0).all())
    s.fetche(pg, ipmin=pg.np + 1, np=0)  # an empty slice is allowed
    with pytest.raises(ValueError):
        s.fetche(pg, ipmin=0, np=10)
    with pytest.raises(ValueError):
        s.fetche(pg, ipmin=pg.np - 5, np=10)
    with pytest.raises(ValueError):
        s.fetche(ipmin=1, np=10)


def test_advance_bitexact_with_quads_and_pipe():
    from warp_b200 import pic
    cfg, s, p, pg = _setup(100_000)
    rng = np.random.default_rng(11)
    phi = np.asfortranarray(1e3 * rng.standard_normal((s.nx + 3, s.ny + 3, s.nz + 3)))
    s.phi = phi
    from warp_b200.lattice import fodo
    lat = fodo(cfg["quad_gradient"], cfg["quad_length"], cfg["period"])
    s.setlattice(lat)
    czs, cze, cdb, nzl, zlmin, dzl = s._lattice
    dt = pic.timestep(cfg)
    # push particles near the wall too
    p2 = {k: v.copy() for k, v in p.items()}
    p2["x"][:1000] *= 8.6
    from warp_b200.particles import ParticleGroup
    pg = ParticleGroup(p2, w=1.0)
    for _ in range(3):
        ex, ey, ez = oracle.sete(phi, p2["x"], p2["y"], p2["z"], s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin)
        oracle.push_fullv(p2, ex, ey, ez, pg.q, pg.m, dt, (czs, cze, cdb), zlmin, dzl, s.zmmin, s.zmmax,
                          cfg["pipe_radius"])
        s.advance(pg, dt, prwall=cfg["pipe_radius"])
    got = pg.to_numpy()
    lost = p2["gaminv"] == 0
    assert lost.sum() > 0
    assert np.array_equal(got["gaminv"], p2["gaminv"])
    for k in ("x", "y", "z", "ux", "uy", "uz"):
        # lost particles are frozen at the step they were lost
        assert np.array_equal(got[k], p2[k]), k


def test_halfv_fullv_synchv_sequence_bitexact():
    """A run as padvnc3d orders it: halfv after loading, fullv steps, and a
    synchv that brings the velocities back to the positions' time."""
    from warp_b200 import pic
    from warp_b200.lattice import fodo
    from warp_b200.particles import ParticleGroup
    cfg, s, p, _ = _setup(50_000)
    rng = np.random.default_rng(12)
    phi = np.asfortranarray(1e3 * rng.standard_normal((s.nx + 3, s.ny + 3, s.nz + 3)))
    s.phi = phi
    s.setlattice(fodo(cfg["quad_gradient"], cfg["quad_length"], cfg["period"]))
    czs, cze, cdb, nzl, zlmin, dzl = s._lattice
    dt = pic.timestep(cfg)
    p2 = {k: v.copy() for k, v in p.items()}
    pg = ParticleGroup(p2, w=1.0)
    for center in ("halfv", "fullv", "fullv", "synchv"):
        ex, ey, ez = oracle.sete(phi, p2["x"], p2["y"], p2["z"], s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin)
        oracle.push(p2, ex, ey, ez, pg.q, pg.m, dt, (czs, cze, cdb), zlmin, dzl, s.zmmin, s.zmmax,
                    cfg["pipe_radius"], center=center)
        s.advance(pg, dt, prwall=cfg["pipe_radius"], center=center)
        got = pg.to_numpy()
        for k in ("x", "y", "z", "ux", "uy", "uz", "gaminv"):
            assert np.array_equal(got[k], p2[k]), (center, k)
    # synchv moves no particle
    x = pg.x.clone()
    s.advance(pg, dt, center="synchv")
    assert torch.equal(pg.x, x)


def test_halfv_then_synchv_is_one_half_kick_each_way():
    """With E only (no lattice): halfv with dt = 0 changes nothing, and
    synchv is exactly one half E kick u + E q (dt/2) / m."""
    from warp_b200 import pic
    from warp_b200.particles import ParticleGroup
    cfg, s, p, _ = _setup(20_000)
    rng = np.random.default_rng(13)
    s.phi = np.asfortranarray(1e3 * rng.standard_normal((s.nx + 3, s.ny + 3, s.nz + 3)))
    dt = pic.timestep(cfg)
    pg = ParticleGroup({k: v.copy() for k, v in p.items()}, w=1.0, with_fields=True)
    s.fetche(pg)
    e0 = (pg.ex.clone(), pg.ey.clone())
    u0 = (pg.ux.clone(), pg.uy.clone())
    s.advance(pg, 0.0, center="halfv")  # dt = 0: no kick, no drift
    assert torch.equal(pg.ux, u0[0]) and torch.equal(pg.uy, u0[1])
    s.advance(pg, dt, center="synchv")  # half kick at the unchanged positions
    cst = pg.q * (0.5 * dt) / pg.m
    assert torch.equal(pg.ux, u0[0] + e0[0] * cst) and torch.equal(pg.uy, u0[1] + e0[1] * cst)


def test_unknown_center_is_rejected():
    cfg, s, p, pg = _setup(1000)
    with pytest.raises(ValueError):
        s.advance(pg, 1e-9, center="gen")
    from warp_b200 import _lib
    import ctypes
    prm = _lib.PushParams(1e-9, 1e30, 0., 0., 0, 7)
    st = pg.cstruct()
    assert _lib.lib.wg_advance(s._h, ctypes.byref(st), ctypes.byref(prm)) == -1


def test_moments_match_oracle():
    cfg, s, p, pg = _setup(300_000)
    p["gaminv"][::13] = 0.0
    pg.gaminv.copy_(torch.as_tensor(p["gaminv"]))
    m = s.moments(pg)
    r = oracle.moments(p)
    assert m["n"] == r["n"]
    for k in ("xbar", "ybar"):
        assert m[k] == pytest.approx(r[k], rel=1e-9, abs=1e-15)
    for k in ("xrms", "yrms", "epsx", "epsy"):
        assert m[k] == pytest.approx(r[k], rel=1e-11)
