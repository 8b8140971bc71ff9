"""Pins the oracle's multigrid against the reference's known-answer test
(warp_test/MutltiGrid3D_test.py): every boundary combination must reach
max error < 1e-10 at mgtol = 1e-12 without hitting mgmaxiters."""
import pytest

from oracle import oracle
from tests import mgkat

COMBOS = mgkat.boundary_combos()


def test_combo_count():
    # 5 distinct choices per axis pair: 00, 01, 10, 11, 22
    assert len(COMBOS) == 125


@pytest.mark.parametrize("bounds", COMBOS, ids=["".join(map(str, b)) for b in COMBOS])
def test_oracle_mg_kat(bounds):
    dx, dy, dz, *_ = mgkat.mesh()
    rho, phi, expected = mgkat.setup(bounds, oracle.eps0())
    iters, err = oracle.mgsolve(phi, rho, dx, dy, dz, bounds, mgtol=1e-12)
    assert iters < 100
    assert mgkat.error(phi, expected, bounds) < 1e-10
