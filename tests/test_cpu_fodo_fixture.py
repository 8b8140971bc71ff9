"""The long-run FODO fixtures (tests/golden/fodo_long_run.npz, 20000
particles, and fodo_long_run_200k.npz, 200000) are what the oracle computes:
their first two lattice periods are recomputed here bit for bit (the
oracle's threaded loops sum in a fixed order), and the particles drawn by
the CPU generator are the fixtures'."""
import os

import numpy as np
import pytest

from tests import fodo_setup as F

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", ["fodo_long_run.npz", "fodo_long_run_200k.npz"])
def test_fixture_first_two_periods_recomputed_by_the_oracle(name):
    g = np.load(os.path.join(GOLDEN, name))
    npart, seed, mgtol = int(g["npart"]), int(g["seed"]), float(g["mgtol"])
    assert np.array_equal(F.host_beam(npart, seed)["x"][:8], g["x0"])
    r = F.oracle_run(npart, 2 * F.STEPS_PER_PERIOD, seed, mgtol)
    for k in ("step", "epsx", "epsy", "live"):
        assert np.array_equal(r[k], g[k][:2]), k
    assert np.array_equal(r["vcycles"], g["vcycles"][:2 * F.STEPS_PER_PERIOD + 1])
    # the fixture covers 20 periods with beam kept
    assert len(g["step"]) == 20 and g["step"][-1] == 1000
    assert g["live"][-1] >= 0.98 * npart
