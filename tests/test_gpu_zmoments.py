"""getzmmnt moment sums on the B200 (wg_zmoments) against the oracle, and
the moments a synchv step records. The GPU adds in an unfixed order, so the
sums agree to rounding: 1e-12 of each moment's largest magnitude."""
import numpy as np
import pytest
import torch

from oracle import oracle
from tests import gpu_helpers as H

pytestmark = pytest.mark.gpu


def _solver():
    return H.make_solver(16, 16, 32, (-0.04, -0.04, 0.0), (0.04, 0.04, 1.0), (0, 0, 0, 0, 2, 2))


def _beam(n, seed=0):
    rng = np.random.default_rng(seed)
    p = {"x": rng.normal(1e-4, 2e-3, n), "y": rng.normal(-2e-4, 1e-3, n), "z": rng.uniform(-0.1, 1.1, n),
         "ux": rng.normal(0, 3e4, n), "uy": rng.normal(0, 2e4, n), "uz": rng.normal(1.4e7, 1e4, n),
         "gaminv": np.ones(n)}
    p["gaminv"][::17] = 0.0
    po = {k: p[k] + rng.normal(0, 50.0, n) for k in ("ux", "uy", "uz")}
    return p, po


@pytest.mark.parametrize("nzmmnt", [1, 64, 512, 1000])
def test_zmoment_sums_match_oracle(nzmmnt):
    """nzmmnt 1000 is past the shared-memory grid (global accumulation)."""
    from warp_b200.particles import ParticleGroup
    s = _solver()
    p, po = _beam(200_000, seed=nzmmnt)
    pg = ParticleGroup(p, w=1.0)
    uold = tuple(torch.as_tensor(po[k], device="cuda") for k in ("ux", "uy", "uz"))
    g, zm = s.zmoments(pg, uold, 1e-9, 0.0, 1.0, nzmmnt, zmmntdtextmax=0.8)
    og, ozm = oracle.zmoments(p, po, 1e-9, 0.0, 1.0, nzmmnt, zmmntdtextmax=0.8)
    assert np.all(np.abs(g - og) <= 1e-12 * np.abs(og) + 1e-300)
    scale = np.abs(ozm).max(axis=0)
    assert np.all(np.abs(zm - ozm) <= 1e-12 * scale)
    assert g[0] == og[0]


def test_synchv_records_moments_history():
    from warp_b200 import pic
    from warp_b200.diagnostics import finalize
    cfg = pic.workload("A")
    run = pic.ESPIC(cfg, tolkind="relres")
    run.generate()
    run.step(3)
    p_before = run.pgroup.to_numpy()
    out = run.synchv(nzmmnt=32)
    assert run.vsync and len(run.history) == 1 and out["it"] == 3
    p_after = run.pgroup.to_numpy()
    og, ozm = oracle.zmoments(p_after, {k: p_before[k] for k in ("ux", "uy", "uz")}, 0.5 * run.dt,
                              cfg["zmmin"], cfg["zmmax"], 32)
    ref = finalize(ozm, "z")
    for k in ("pnumz", "xbarz", "xrmsz", "yrmsz", "epsxz", "epsyz"):
        assert np.allclose(out[k], ref[k], rtol=1e-9, atol=1e-15), k
    refg = finalize(og)
    for k in ("pnum", "xrms", "epsx", "epsy", "vzbar"):
        assert out[k] == pytest.approx(refg[k], rel=1e-9), k
    # the global x rms agrees with the plain moments kernel
    assert out["xrms"] == pytest.approx(run.moments()["xrms"], rel=1e-9)
    assert run.synchv(nzmmnt=32) is None  # already in step
