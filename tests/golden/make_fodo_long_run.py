"""Writes fodo_long_run.npz: the oracle's FODO run (the configuration of
tests/fodo_setup.py) with 20000 particles over 1000 steps (20 lattice
periods), multigrid to max |dphi| <= 1e-6 V, recording the emittances and the
live-particle count after every period and the V-cycles of every solve. It
also stores the first initial x values, so that a test can check that the
particles it draws are the ones the fixture was made from.

Run from the repository root: python tests/golden/make_fodo_long_run.py
(about 30 s on 16 host threads)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests import fodo_setup as F  # noqa: E402

NPART, NSTEPS, SEED, MGTOL = 20_000, 1000, 72, 1e-6


def main():
    r = F.oracle_run(NPART, NSTEPS, SEED, MGTOL)
    x0 = F.host_beam(NPART, SEED)["x"][:8]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "fodo_long_run.npz")
    np.savez(out, npart=NPART, nsteps=NSTEPS, seed=SEED, mgtol=MGTOL, x0=x0, **r)
    print("wrote %s: epsx %.6e -> %.6e, live %d, V-cycles %d" % (out, r["epsx"][0], r["epsx"][-1], r["live"][-1],
                                                                 r["vcycles"].sum()))


if __name__ == "__main__":
    main()
