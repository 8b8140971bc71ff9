"""Field-solver registry and the interpreter-level helpers of
scripts/fieldsolver.py: registersolver (:173-181), getregisteredsolver,
unregistersolver, loadrho (:11), fieldsolve (:49) and fetche (:95).

In WARP, registersolver sets top.fstype = 12 and the Fortran step then calls
loadrhoregistered / fieldsolregistered / fetcheregistered, which dispatch to
solver.loadrho(), solver.solve() and solver.fetche() (:206-257). The same
dispatch is done here for decks driven from Python (warp_b200.pic.step).
"""

_registeredsolvers = []


class FieldSolver:
    """Base class of registered solvers (scripts/fieldsolver.py:378).
    Subclasses implement loadrho, solve, fetche."""

    def loadrho(self, pgroups=None, lzero=True, lfinalize_rho=True):
        raise NotImplementedError

    def solve(self, iwhich=0):
        raise NotImplementedError

    def fetche(self, pgroup=None):
        raise NotImplementedError


def registersolver(solver):
    """Registers a field solver; the PIC step then uses it for the field
    solve (top.fstype = 12 in the reference)."""
    if not isinstance(solver, FieldSolver):
        raise TypeError("registersolver: expected a FieldSolver instance")
    if solver not in _registeredsolvers:
        _registeredsolvers.append(solver)


def unregistersolver(solver=None, i=None):
    if solver is not None:
        _registeredsolvers.remove(solver)
    elif i is not None:
        del _registeredsolvers[i]
    else:
        raise ValueError("unregistersolver: give solver or i")


def getregisteredsolver(i=0):
    return _registeredsolvers[i] if len(_registeredsolvers) > i else None


def getregisteredsolvers():
    return list(_registeredsolvers)


def _solver():
    s = getregisteredsolver()
    if s is None:
        raise RuntimeError("no field solver registered (call registersolver first)")
    return s


def loadrho(pgroup=None, lzero=True, lfinalize_rho=True):
    """Deposits the charge of pgroup (or all groups known to the solver)."""
    return _solver().loadrho(pgroups=None if pgroup is None else [pgroup], lzero=lzero,
                             lfinalize_rho=lfinalize_rho)


def fieldsolve(iwhich=0):
    """Field solve of every registered solver (fieldsolregistered)."""
    if iwhich > 0:
        return
    for s in _registeredsolvers:
        s.solve(iwhich)


fieldsol = fieldsolve


def fetche(pgroup=None):
    return _solver().fetche(pgroup)
