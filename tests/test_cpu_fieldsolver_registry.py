"""The registered-solver dispatch of scripts/fieldsolver.py (registersolver
:173-181, loadrho :11, fieldsolve :49, fetche :95, and the Fortran-side
loadrhoregistered / fieldsolregistered / fetcheregistered :206-257) on a
stand-in solver: what a deck calls reaches the registered solver with the
reference's arguments, and misuse raises."""
import pytest

from warp_b200 import fieldsolver as fs


class _Recorder(fs.FieldSolver):
    def __init__(self):
        self.calls = []

    def loadrho(self, pgroups=None, lzero=True, lfinalize_rho=True):
        self.calls.append(("loadrho", pgroups, lzero, lfinalize_rho))

    def solve(self, iwhich=0):
        self.calls.append(("solve", iwhich))

    def fetche(self, pgroup=None):
        self.calls.append(("fetche", pgroup))
        return "E"


@pytest.fixture(autouse=True)
def _clean_registry():
    saved = list(fs._registeredsolvers)
    fs._registeredsolvers.clear()
    yield
    fs._registeredsolvers[:] = saved


def test_dispatch_reaches_the_registered_solver():
    s = _Recorder()
    fs.registersolver(s)
    fs.registersolver(s)  # registering twice keeps one entry
    assert fs.getregisteredsolvers() == [s] and fs.getregisteredsolver() is s
    fs.loadrho()
    fs.loadrho("pg", lzero=False)
    fs.fieldsolve()
    fs.fieldsolve(1)  # only iwhich 0 solves
    assert fs.fetche("pg") == "E"
    assert s.calls == [("loadrho", None, True, True), ("loadrho", ["pg"], False, True), ("solve", 0),
                       ("fetche", "pg")]


def test_every_registered_solver_solves():
    a, b = _Recorder(), _Recorder()
    fs.registersolver(a)
    fs.registersolver(b)
    fs.fieldsol()
    assert a.calls == [("solve", 0)] and b.calls == [("solve", 0)]
    fs.unregistersolver(a)
    assert fs.getregisteredsolvers() == [b]
    fs.unregistersolver(i=0)
    assert fs.getregisteredsolver() is None


def test_misuse_raises():
    with pytest.raises(TypeError):
        fs.registersolver(object())
    with pytest.raises(RuntimeError):
        fs.loadrho()
    with pytest.raises(RuntimeError):
        fs.fetche()
    with pytest.raises(ValueError):
        fs.unregistersolver()
    with pytest.raises(NotImplementedError):
        fs.FieldSolver().solve()


def test_lprecalccoeffs_is_refused_clearly():
    """A deck that sets lprecalccoeffs gets NotImplementedError with the
    reason, before any device work."""
    import pytest
    from warp_b200.multigrid import MultiGridB200
    with pytest.raises(NotImplementedError, match="lprecalccoeffs"):
        MultiGridB200(8, 8, 8, 0., 1., 0., 1., 0., 1., lprecalccoeffs=True)
