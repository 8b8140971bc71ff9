"""The PIC step of warp_b200.pic.ESPIC run on the CPU oracle.

TEST INFRASTRUCTURE ONLY: used by tests/ and by bench.py's CPU legs (the
reference arm and the cpu_baseline) as the reference's arithmetic on the
host cores. The warp_b200 package never imports it, and it loads no CUDA
library: the workload, beam and lattice come from warp_b200.workloads and
warp_b200.lattice, which are plain numpy.

One step is the order of step3d (pywarp90/w3d.F:511-986): gather and push
(sete3d + padvnc3d, halfv on the first step after loading, fullv after),
deposit (setrho3d + applyrhoboundaryconditions3d) and the multigrid solve
(multigrid3dsolve) warm-started from the previous phi. With
tolkind "relres" the solve runs V-cycles until
max|rhs - A phi| / max|rhs| <= mgtol, testing before every V-cycle as the
GPU solver does; with "mgerror" it is the reference's own max|dphi| test.
"""
import numpy as np

from oracle import oracle

BOUNDS = (0, 0, 0, 0, 2, 2)


class OracleESPIC:
    def __init__(self, cfg, tolkind="relres", mgtol=1e-6, mgmaxiters=100, particles=None, npart=None, w=None,
                 phi=None, vsync=True):
        from warp_b200.constants import echarge, proton_mass
        from warp_b200.lattice import fodo
        from warp_b200.workloads import beam_weight, semigaussian, timestep
        c = self.cfg = cfg
        self.nx, self.ny, self.nz = c["nx"], c["ny"], c["nz"]
        self.dx = (c["xmmax"] - c["xmmin"]) / self.nx
        self.dy = (c["ymmax"] - c["ymmin"]) / self.ny
        self.dz = (c["zmmax"] - c["zmmin"]) / self.nz
        self.mins = (c["xmmin"], c["ymmin"], c["zmmin"])
        self.tolkind, self.mgtol, self.mgmaxiters = tolkind, float(mgtol), int(mgmaxiters)
        if particles is None:
            n = c["npart"] if npart is None else int(npart)
            particles = semigaussian(n, seed=c["seed"], radius=c["radius"], mismatch=c["mismatch"],
                                     angle_rms=c["angle_rms"], zmin=c["zmmin"], zmax=c["zmmax"],
                                     ekin_ev=c["ekin_ev"])
        self.p = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in particles.items()}
        self.q, self.m = echarge, proton_mass
        # the weight of the full workload's beam current, spread over the
        # particles actually loaded (or the weight of a run being continued)
        self.w = (beam_weight(c["current"], c["zmmax"] - c["zmmin"], len(self.p["x"]), ekin_ev=c["ekin_ev"])
                  if w is None else float(w))
        self.dt = timestep(c)
        lat = fodo(c["quad_gradient"], c["quad_length"], c["period"])
        self.zlmin, self.dzl = c["zmmin"], self.dz
        nzl = int(round((c["zmmax"] - self.zlmin) / self.dzl)) + 1
        self.tables = tuple(np.ascontiguousarray(a) for a in lat.tables(self.zlmin, self.dzl, nzl))
        oc = oracle.Conductors(self.nx, self.ny, self.nz, self.dx, self.dy, self.dz, *self.mins)
        zc = 0.5 * (c["zmmin"] + c["zmmax"])
        oc.add_shape("ZCylinderOut", c["pipe_radius"], 100.0, 0.0, 0., 0., zc, 1)
        if c.get("rods"):
            d = c["rod_center"]
            for (x, y, v) in ((d, 0., c["rod_voltage"]), (-d, 0., c["rod_voltage"]),
                              (0., d, -c["rod_voltage"]), (0., -d, -c["rod_voltage"])):
                oc.add_shape("ZCylinder", c["rod_radius"], 100.0, v, x, y, zc, 1)
        oc.finalize()
        self.cond = oc
        self.phi = (np.zeros((self.nx + 3, self.ny + 3, self.nz + 3), order="F") if phi is None
                    else np.asfortranarray(phi, dtype=np.float64))
        self.rho = np.zeros((self.nx + 1, self.ny + 1, self.nz + 1), order="F")
        # velocities at the positions' time (the next step is halfv)
        self.vsync = bool(vsync)
        self.it = 0
        self.mgiters = 0
        self.relres = -1.0

    def deposit(self):
        self.rho[...] = 0.0
        p = self.p
        oracle.setrho(self.rho, p["x"], p["y"], p["z"], self.q, self.w, self.dx, self.dy, self.dz, *self.mins,
                      gaminv=p["gaminv"])
        oracle.rhobc(self.rho, BOUNDS)

    def solve(self):
        """Returns the V-cycles done."""
        if self.tolkind == "mgerror":
            it, _ = oracle.mgsolve(self.phi, self.rho, self.dx, self.dy, self.dz, BOUNDS, conductors=self.cond,
                                   mgtol=self.mgtol, mgmaxiters=self.mgmaxiters)
            self.mgiters = it
            return it
        it = 0
        while True:
            self.relres = oracle.relresidual(self.phi, self.rho, self.dx, self.dy, self.dz, BOUNDS, self.cond)
            if self.relres <= self.mgtol or it >= self.mgmaxiters:
                break
            oracle.mgsolve(self.phi, self.rho, self.dx, self.dy, self.dz, BOUNDS, conductors=self.cond, mgtol=0.0,
                           mgmaxiters=1)
            it += 1
        self.mgiters = it
        return it

    def generate(self):
        self.deposit()
        return self.solve()

    def advance(self):
        p, c = self.p, self.cfg
        ex, ey, ez = oracle.sete(self.phi, p["x"], p["y"], p["z"], self.dx, self.dy, self.dz, *self.mins)
        oracle.push(p, ex, ey, ez, self.q, self.m, self.dt, self.tables, self.zlmin, self.dzl, c["zmmin"],
                    c["zmmax"], c["pipe_radius"], center="halfv" if self.vsync else "fullv")
        self.vsync = False

    def step(self):
        """One PIC step; returns the V-cycles of its solve."""
        self.advance()
        self.deposit()
        self.it += 1
        return self.solve()
