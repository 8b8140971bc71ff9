"""getzmmnt's moment sums (itask = 2, ifzmmnt = 2, top.F:814-1160) in the
oracle against an independent numpy restatement, and the finalization
(itask = 3, top.F:1317-1700) on beams with known moments."""
import numpy as np
import pytest

from oracle import oracle
from warp_b200 import diagnostics as D


def _beam(n, seed=0):
    rng = np.random.default_rng(seed)
    p = {"x": rng.normal(1e-4, 2e-3, n), "y": rng.normal(-2e-4, 1e-3, n), "z": rng.uniform(-0.1, 1.1, n),
         "ux": rng.normal(0, 3e4, n), "uy": rng.normal(0, 2e4, n), "uz": rng.normal(1.4e7, 1e4, n),
         "gaminv": np.ones(n)}
    p["gaminv"][::17] = 0.0  # lost particles
    po = {k: p[k] + rng.normal(0, 50.0, n) for k in ("ux", "uy", "uz")}
    return p, po


def test_oracle_sums_match_numpy_restatement():
    p, po = _beam(20000)
    a0, a = oracle.zmoments(p, po, 1e-9, 0.0, 1.0, 32, zmmntdtextmax=0.7)
    b0, b = D.zmoment_sums_host(p, po, 1e-9, 0.0, 1.0, 32, zmmntdtextmax=0.7)
    assert np.allclose(a0, b0, rtol=1e-12, atol=0)
    scale = np.abs(b).max(axis=0) + 1e-300
    assert np.all(np.abs(a - b) <= 1e-12 * scale)
    # every live particle in range adds weight 1 over its two planes
    live = p["gaminv"] != 0
    inr = live & (p["z"] >= 0.0) & (p["z"] < 1.0)
    assert a[:, 0].sum() == pytest.approx(inr.sum(), rel=1e-12)
    assert a0[0] == live.sum()


def test_constant_velocity_particle_lands_on_the_planes():
    """With no velocity change the extrapolation is a straight line: each
    plane sees the particle at the plane's z."""
    p = {"x": np.array([1e-3]), "y": np.array([2e-3]), "z": np.array([0.37]), "ux": np.array([1e4]),
         "uy": np.array([-2e4]), "uz": np.array([1e7]), "gaminv": np.ones(1)}
    po = {k: p[k].copy() for k in ("ux", "uy", "uz")}
    z0, zm = oracle.zmoments(p, po, 1e-9, 0.0, 1.0, 10)
    m = D.finalize(zm, "z")
    assert m["zbarz"][3] == pytest.approx(0.3, rel=1e-12)
    assert m["zbarz"][4] == pytest.approx(0.4, rel=1e-12)
    assert m["pnumz"][3] == pytest.approx(0.3, rel=1e-12) and m["pnumz"][4] == pytest.approx(0.7, rel=1e-12)
    assert m["xbarz"][3] == pytest.approx(1e-3 + 1e4 * (0.3 - 0.37) / 1e7, rel=1e-12)


def test_finalize_rms_and_emittance_of_known_beams():
    rng = np.random.default_rng(3)
    n = 400000
    x = rng.normal(0, 2e-3, n)
    xp = rng.normal(0, 1e-3, n)
    uz = np.full(n, 1e7)
    p = {"x": x, "y": 0.5 * x, "z": rng.uniform(0, 1, n), "ux": xp * uz, "uy": np.zeros(n), "uz": uz,
         "gaminv": np.ones(n)}
    g, _ = oracle.zmoments(p, {k: p[k] for k in ("ux", "uy", "uz")}, 1e-9, 0.0, 1.0, 4)
    m = D.finalize(g)
    assert m["xrms"] == pytest.approx(np.std(x), rel=1e-9)
    assert m["epsx"] == pytest.approx(4 * np.std(x) * np.std(xp), rel=2e-2)
    # y = x/2 with y' = 0: zero y emittance
    assert m["epsy"] == pytest.approx(0.0, abs=1e-12)
    # a fully correlated phase space has zero emittance
    p["ux"] = 0.3 * x * uz
    g, _ = oracle.zmoments(p, {k: p[k] for k in ("ux", "uy", "uz")}, 1e-9, 0.0, 1.0, 4)
    assert D.finalize(g)["epsx"] <= 1e-9 * D.finalize(g)["xrms"] * 0.3 * 4
