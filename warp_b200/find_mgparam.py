"""find_mgparam (scripts/find_mgparam.py:28-237): tunes the over-relaxation
parameter mgparam and the numbers of down and up passes of a multigrid
solver for the shortest field solve on the problem it currently holds.

The search is the reference's:
- the outer loop raises downpasses and uppasses together while the timed
  solve gets faster, and steps back once it does not (:83-102);
- the inner loop (_find_mgparam, :171-237) walks mgparam in steps of 0.05,
  reversing and halving the step whenever a solve needs more V-cycles,
  until two solves in a row need the same number or 20 tries pass; an
  mgparam that leaves (0.01, 2] restarts near 1.9;
- every timed solve starts from phi = 0 on the nodes the solver updates
  (boundary planes of Dirichlet faces keep their values), or from the saved
  phi with lsavephi (:119-150);
- when a solve hits mgmaxiters, mgtol is loosened to ten times the reached
  error for the search and restored at the end (:71-82, :116).

The solver only needs the MultiGrid3D attributes (mgparam, downpasses,
uppasses, mgtol, mgiters, mgerror, mgmaxiters, bounds, nx, ny, nz), a phi
array with one guard node on each side, and solve(). The clock and the
random restart are arguments so that the search itself can be checked
without a GPU.
"""
import time

import numpy as np


def _zero_updated_nodes(solver):
    b = solver.bounds
    ixmin, ixmax = (0 if b[0] > 0 else 1), (solver.nx if b[1] > 0 else solver.nx - 1)
    iymin, iymax = (0 if b[2] > 0 else 1), (solver.ny if b[3] > 0 else solver.ny - 1)
    izmin, izmax = (0 if b[4] > 0 else 1), (solver.nz if b[5] > 0 else solver.nz - 1)
    solver.phi[ixmin + 1:ixmax + 2, iymin + 1:iymax + 2, izmin + 1:izmax + 2] = 0.0


def field_solve(solver, phisave, clock=time.perf_counter):
    """One timed solve from phi = 0 (phisave None) or from phisave."""
    if phisave is None:
        _zero_updated_nodes(solver)
    else:
        solver.phi[...] = phisave
    t0 = clock()
    solver.solve()
    return clock() - t0


def _find_mgparam(solver, phisave, clock, rng, log):
    if solver.mgparam <= 0.0:
        solver.mgparam = max(1.0, 2.0 + solver.mgparam)
    if solver.mgparam > 2.0:
        solver.mgparam = max(1.0, 4.0 - solver.mgparam)
    fstime = field_solve(solver, phisave, clock)
    mgparam_prev, mgiters_prev = solver.mgparam, solver.mgiters
    sincr = 0.05
    iters = 0  # forces one pass of the loop, as the reference's mgiters = 0
    solver.mgparam = solver.mgparam + sincr
    icount = 0
    while mgiters_prev != iters and icount < 20:
        log("Best parameter so far = %f" % solver.mgparam)
        fstime = field_solve(solver, phisave, clock)
        iters = solver.mgiters
        if iters > mgiters_prev:
            sincr = -sincr / 2.0
            solver.mgparam = mgparam_prev + sincr
        elif iters < mgiters_prev:
            iters, mgiters_prev = mgiters_prev, iters
            mgparam_prev = solver.mgparam
            solver.mgparam = mgparam_prev + sincr
        if solver.mgparam <= 0.01 or solver.mgparam > 2.0:
            solver.mgparam = 1.9 + rng.random() * 0.05
            sincr = 0.01
        icount += 1
    if icount == 20:
        log("Warning: maximum number of iterations reached; mgparam may not be optimal.")
    return fstime


def find_mgparam(solver, lsavephi=False, resetpasses=0, clock=time.perf_counter, seed=0, log=print):
    """Sets solver.mgparam, downpasses and uppasses to the fastest values
    found; returns the best solve time. The solver's phi holds the last
    trial solve afterwards (the saved phi with lsavephi, re-solved)."""
    rng = np.random.default_rng(seed)
    phisave = solver.phi.clone() if lsavephi and hasattr(solver.phi, "clone") else (
        np.array(solver.phi, copy=True) if lsavephi else None)
    if resetpasses:
        solver.downpasses = 1
        solver.uppasses = 1
    solver.downpasses = max(1, solver.downpasses)
    solver.uppasses = max(1, solver.uppasses)
    nexttime = field_solve(solver, phisave, clock)
    prevtime = 2 * nexttime
    savemgtol = solver.mgtol
    if solver.mgiters == solver.mgmaxiters:
        solver.mgtol = 10 * solver.mgerror
        nexttime = field_solve(solver, phisave, clock)
        prevtime = 2 * nexttime
    while nexttime < prevtime:
        prevparam = solver.mgparam
        prevtime = nexttime
        nexttime = _find_mgparam(solver, phisave, clock, rng, log)
        log("Field solve time = %g; mgparam = %g; downpasses = %d; uppasses = %d" % (
            nexttime, solver.mgparam, solver.downpasses, solver.uppasses))
        if nexttime < prevtime:
            solver.downpasses += 1
            solver.uppasses += 1
        else:
            solver.mgparam = prevparam
            solver.downpasses = max(1, solver.downpasses - 1)
            solver.uppasses = max(1, solver.uppasses - 1)
    if solver.mgiters == solver.mgmaxiters:
        log("Notice: the maximum number of iterations has been reached, so the values found are unlikely "
            "to be optimal.")
    else:
        log("Optimized: field solve time = %g; mgparam = %g; downpasses = %d; uppasses = %d" % (
            prevtime, solver.mgparam, solver.downpasses, solver.uppasses))
    solver.mgtol = savemgtol
    return prevtime
