"""The mgparam search of find_mgparam (scripts/find_mgparam.py:28-237) on a
stand-in solver whose V-cycle count is a known function of mgparam and of
the passes, with a simulated clock: the search ends at the optimum the
reference's walk reaches, trials start from phi = 0 on the updated nodes
only, and a loosened mgtol is restored."""
import numpy as np

from warp_b200.find_mgparam import find_mgparam


class FakeSolver:
    def __init__(self, bounds=(0, 0, 0, 0, 2, 2), best=1.72, cost_per_pass=1.0):
        self.nx, self.ny, self.nz = 6, 5, 8
        self.bounds = list(bounds)
        self.mgparam, self.downpasses, self.uppasses = 1.2, 1, 1
        self.mgtol, self.mgiters, self.mgmaxiters, self.mgerror = 1e-6, 0, 100, 0.0
        self.phi = np.full((self.nx + 3, self.ny + 3, self.nz + 3), 5.0)
        self.best, self.cost = best, cost_per_pass
        self.now = 0.0
        self.starts = []
        self.solves = 0

    def clock(self):
        return self.now

    def solve(self):
        self.starts.append(self.phi.copy())
        self.solves += 1
        passes = self.downpasses + self.uppasses
        # V-cycles fall with more passes, each V-cycle costs more
        self.mgiters = int(round(8 + 300 * (self.mgparam - self.best) ** 2 + 12.0 / passes))
        self.mgerror = 1e-7
        self.now += self.mgiters * (passes + 2) * self.cost


def test_search_finds_the_fast_mgparam_and_passes():
    s = FakeSolver()
    t = find_mgparam(s, resetpasses=1, clock=s.clock, log=lambda *a: None)
    assert abs(s.mgparam - s.best) < 0.1
    assert s.mgiters <= 9 + 12
    assert (s.downpasses, s.uppasses) in ((1, 1), (2, 2))
    assert t > 0 and s.mgtol == 1e-6


def test_trials_start_from_zero_on_the_updated_nodes():
    s = FakeSolver(bounds=(0, 0, 1, 1, 2, 2))
    find_mgparam(s, clock=s.clock, log=lambda *a: None)
    start = s.starts[0]
    # Dirichlet x faces keep their values; Neumann y and periodic z faces are updated
    assert np.all(start[1, :, :] == 5.0) and np.all(start[s.nx + 1, :, :] == 5.0)
    assert np.all(start[2:s.nx + 1, 1:s.ny + 2, 1:s.nz + 2] == 0.0)
    # guard nodes are left alone
    assert np.all(start[0] == 5.0) and np.all(start[:, 0] == 5.0)


def test_lsavephi_restarts_every_trial_from_the_saved_phi():
    s = FakeSolver()
    s.phi[...] = np.arange(s.phi.size, dtype=float).reshape(s.phi.shape)
    saved = s.phi.copy()
    find_mgparam(s, lsavephi=True, clock=s.clock, log=lambda *a: None)
    assert len(s.starts) > 3
    assert all(np.array_equal(st, saved) for st in s.starts)


def test_mgtol_loosened_at_mgmaxiters_and_restored():
    s = FakeSolver(best=5.0)  # far optimum: the first solve hits mgmaxiters
    s.mgmaxiters = 50
    seen = []
    solve = s.solve

    def record():
        seen.append(s.mgtol)
        solve()
        s.mgiters = min(s.mgiters, s.mgmaxiters)
    s.solve = record
    find_mgparam(s, clock=s.clock, log=lambda *a: None)
    assert seen[0] == 1e-6 and seen[1] == 10 * 1e-7
    assert s.mgtol == 1e-6
    assert 0.01 < s.mgparam <= 2.0
