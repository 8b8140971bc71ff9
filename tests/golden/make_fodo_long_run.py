"""Writes the oracle's FODO runs (the configuration of tests/fodo_setup.py)
over 1000 steps (20 lattice periods), multigrid to max |dphi| <= 1e-6 V,
recording the emittances and the live-particle count after every period and
the V-cycles of every solve. Each file also stores the first initial x
values, so that a test can check that the particles it draws are the ones
the fixture was made from.

- fodo_long_run.npz: 20000 particles (about 1.5 per occupied cell, the
  particle count of the reference's own FODO test), about 30 s on 16 host
  threads;
- fodo_long_run_200k.npz: 200000 particles (about 15 per occupied cell),
  about 100 s on 8 host threads.

Run from the repository root: python tests/golden/make_fodo_long_run.py
[20000|200000] (both when no count is given)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests import fodo_setup as F  # noqa: E402

NSTEPS, SEED, MGTOL = 1000, 72, 1e-6
FILES = {20_000: "fodo_long_run.npz", 200_000: "fodo_long_run_200k.npz"}


def main(npart):
    r = F.oracle_run(npart, NSTEPS, SEED, MGTOL)
    x0 = F.host_beam(npart, SEED)["x"][:8]
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), FILES[npart])
    np.savez(out, npart=npart, nsteps=NSTEPS, seed=SEED, mgtol=MGTOL, x0=x0, **r)
    print("wrote %s: epsx %.6e -> %.6e, live %d, V-cycles %d" % (out, r["epsx"][0], r["epsx"][-1], r["live"][-1],
                                                                 r["vcycles"].sum()))


if __name__ == "__main__":
    for n in ([int(a) for a in sys.argv[1:]] or sorted(FILES)):
        main(n)
