"""Hard-edge quadrupole lattice (the quad part of scripts/lattice.py Quad /
addnewquad, and of setlattzt, pywarp90/top_lattice.F:1852-2030).

The lattice is a list of quads over one period `zlatperi` starting at
`zlatstrt`; it repeats periodically. `tables()` builds the per-lattice-cell
arrays (cquadzs, cquadze, cquaddb) that applyquad reads: lattice cell iz
(centre zlmin + iz*dzl) is given the quad whose territory contains that
centre, territories being bounded by the midpoints of the drifts between
neighbouring quads (getelemid, top_lattice.F:2369-2440).
"""
import math

import numpy as np


class Quad:
    """Hard-edge magnetic quadrupole: zs..ze, gradient db (T/m)."""

    def __init__(self, zs, ze, db):
        if not ze > zs:
            raise ValueError("Quad needs ze > zs")
        self.zs, self.ze, self.db = float(zs), float(ze), float(db)


class Lattice:
    def __init__(self, quads, zlatperi, zlatstrt=0.0):
        if not quads:
            raise ValueError("Lattice needs at least one quad")
        self.quads = sorted(quads, key=lambda q: q.zs)
        self.zlatperi = float(zlatperi)
        self.zlatstrt = float(zlatstrt)

    def tables(self, zlmin, dzl, nzl):
        zs = [q.zs for q in self.quads]
        ze = [q.ze for q in self.quads]
        db = [q.db for q in self.quads]
        n = len(zs)
        P = self.zlatperi
        czs = np.zeros(nzl + 1)
        cze = np.zeros(nzl + 1)
        cdb = np.zeros(nzl + 1)
        # territory boundaries within one period
        left = [0.5 * (zs[0] + ze[n - 1] - P)] + [0.5 * (zs[k] + ze[k - 1]) for k in range(1, n)]
        right = [0.5 * (ze[k] + zs[k + 1]) for k in range(n - 1)] + [0.5 * (ze[n - 1] + zs[0] + P)]
        for iz in range(nzl + 1):
            zz = zlmin + iz * dzl
            offset = math.floor((zz - self.zlatstrt) / P) * P + self.zlatstrt
            zloc = zz - offset
            if zloc < left[0]:
                # before the first territory: the last quad of the previous period
                best = n - 1
                offset -= P
            elif zloc >= left[0] + P:
                # past the last territory: the first quad of the next period
                best = 0
                offset += P
            else:
                best = next((k for k in range(n) if left[k] <= zloc < right[k]), 0)
            czs[iz] = zs[best] + offset
            cze[iz] = ze[best] + offset
            cdb[iz] = db[best]
        return czs, cze, cdb


def fodo(gradient, quad_length, period, zcenter_first=0.0):
    """FODO cell of hard-edge quads: focusing (+gradient) centred at
    zcenter_first, defocusing (-gradient) half a period later."""
    h = 0.5 * quad_length
    qf = Quad(zcenter_first - h, zcenter_first + h, +gradient)
    qd = Quad(zcenter_first + 0.5 * period - h, zcenter_first + 0.5 * period + h, -gradient)
    return Lattice([qf, qd], zlatperi=period, zlatstrt=0.0)
