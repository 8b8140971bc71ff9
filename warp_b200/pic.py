"""3D electrostatic PIC run on one B200: the step of w3dexe/step3d
(pywarp90/w3d.F:511-986) with the field solve delegated to a registered
MultiGridB200.

Order inside one step (step3d): particle advance with the field of the
previous solve (padvnc3d: gather, quads, leapfrog/Boris, drift), particle
boundaries (periodic z, absorbing pipe), charge deposition (loadrho), field
solve. Loaded velocities are at the positions' time, so the first step is
halfv (w3d.F:780 with lspecial at it == 0) and the steps after it fullv;
ESPIC.synchv() brings the velocities back to the positions' time for
diagnostics, after which the next step is halfv again.

The synthetic workloads (A, B, D, E) are defined in warp_b200.workloads.
"""
import numpy as np

from . import conductors as cond
from .constants import echarge, proton_mass
from .fieldsolver import registersolver
from .lattice import fodo
from .multigrid import MultiGridB200
from .particles import ParticleGroup
from .workloads import (COMMON, WORKLOADS, beam_velocity, beam_weight,  # noqa: F401
                        semigaussian, timestep, workload)


class ESPIC:
    """Sets up solver, conductors, lattice and beam of a workload."""

    def __init__(self, cfg, precision="fp64", tolkind="mgerror", mgtol=1.e-6, mgmaxiters=100, device="cuda",
                 particles=None, sort_interval=0, particle_dtype=None):
        """precision "fp64" is the reference's arithmetic throughout;
        "mixed" runs the V-cycles in FP32 inside FP64 defect correction and
        keeps the particles in FP32 with an FP32 push (particle_dtype, by
        default float32 for "mixed" and float64 for "fp64")."""
        import torch
        if particle_dtype is None:
            particle_dtype = torch.float32 if precision == "mixed" else torch.float64
        self.cfg = cfg
        c = cfg
        self.solver = MultiGridB200(c["nx"], c["ny"], c["nz"], c["xmmin"], c["xmmax"], c["ymmin"], c["ymmax"],
                                    c["zmmin"], c["zmmax"], bounds=(0, 0, 0, 0, 2, 2), precision=precision,
                                    tolkind=tolkind, mgtol=mgtol, mgmaxiters=mgmaxiters, mgverbose=-1,
                                    device=device)
        registersolver(self.solver)
        zc = 0.5 * (c["zmmin"] + c["zmmax"])
        self.solver.installconductor(cond.ZCylinderOut(radius=c["pipe_radius"], length=100.0, zcent=zc))
        if c.get("rods"):
            d = c["rod_center"]
            for (x, y, v) in ((d, 0., c["rod_voltage"]), (-d, 0., c["rod_voltage"]),
                              (0., d, -c["rod_voltage"]), (0., -d, -c["rod_voltage"])):
                self.solver.installconductor(cond.ZCylinder(radius=c["rod_radius"], length=100.0, voltage=v,
                                                            xcent=x, ycent=y, zcent=zc))
        self.lattice = fodo(c["quad_gradient"], c["quad_length"], c["period"])
        self.solver.setlattice(self.lattice)
        self.dt = timestep(c)
        if particles is None:
            particles = semigaussian(c["npart"], seed=c["seed"], radius=c["radius"], mismatch=c["mismatch"],
                                     angle_rms=c["angle_rms"], zmin=c["zmmin"], zmax=c["zmmax"],
                                     ekin_ev=c["ekin_ev"])
        w = beam_weight(c["current"], c["zmmax"] - c["zmmin"], c["npart"], ekin_ev=c["ekin_ev"])
        self.pgroup = ParticleGroup(particles, q=echarge, m=proton_mass, w=w, device=device, dtype=particle_dtype)
        self.solver.addpgroup(self.pgroup)
        self.sort_interval = int(sort_interval)
        # optional learned initial guess (warp_b200.unet.WarmStart): applied
        # to phi after the deposit, before each solve; the multigrid then
        # finishes the solve from it
        self.warmstart = None
        self.it = 0
        # velocities at the positions' time (true after loading and synchv)
        self.vsync = True

    def close(self):
        """Unregisters the run's solver and drops its particles, so that the
        device memory of both is freed once the run object goes (the
        registry of registered solvers would keep them alive)."""
        from .fieldsolver import getregisteredsolvers, unregistersolver
        if self.solver in getregisteredsolvers():
            unregistersolver(self.solver)
        self.solver.pgroups = []
        self.warmstart = None

    def generate(self):
        """Initial deposit and field solve (w3dgen -> step3d("w3dgen"))."""
        if self.sort_interval > 0:
            self.pgroup.sort(self.solver)
        self.solver.loadrho()
        self.solver.solve()

    def _center(self):
        return "halfv" if self.vsync else "fullv"

    def step(self, n=1):
        """n steps of step3d: advance, particle boundaries, loadrho, solve.
        The advance and the deposit run as one pass over the particles
        (MultiGridB200.advance with deposit=True) when this run's group is
        the solver's only species; rho is the same bit for bit."""
        s, pg = self.solver, self.pgroup
        fused = s.pgroups == [pg]
        for _ in range(n):
            if fused:
                s.deposit_begin()
            s.advance(pg, self.dt, prwall=self.cfg["pipe_radius"], center=self._center(), deposit=fused)
            self.vsync = False
            if self.sort_interval > 0 and (self.it + 1) % self.sort_interval == 0:
                # re-sort by cell (and drop lost particles) every sort_interval
                # steps; the fixed-point deposit does not depend on the order
                pg.sort(s)
            if fused:
                s.deposit_end(zero_first=True)
            else:
                s.loadrho()
            if self.warmstart is not None:
                self.warmstart.guess(s)
            s.solve()
            self.it += 1

    def step_host(self, host, nchunks=8):
        """One step of the drop-in mode in which the host owns the particles
        (WARP keeps top.pgroup in host memory); run_host with nsteps = 1."""
        self.run_host(host, 1, nchunks)

    def run_host(self, host, nsteps=1, nchunks=8):
        """nsteps steps of the drop-in mode in which the host owns the
        particles (WARP keeps top.pgroup in host memory, and step(n) runs n
        steps): `host` maps each of x, y, z, ux, uy, uz, gaminv to a pinned
        CPU tensor of the particle group's dtype (float32 in the mixed
        form). Every step reads the arrays from the host and writes the
        advanced particles back.

        The arrays cross PCIe in `nchunks` chunks. Uploads run on one copy
        stream; each chunk is advanced and deposited as soon as it has
        landed, then goes back on a second copy stream, so downloads overlap
        the remaining uploads (PCIe is full duplex). The pieces accumulate in
        one fixed-point deposit, so rho is the same as after step(). The
        uploads of the next step are queued before this step's field solve:
        chunk k goes up as soon as this step has brought chunk k down, so the
        transfers of step n+1 overlap the solve of step n. The host arrays
        are complete once the call returns and the current stream has been
        synchronized; the device state is then the same as after nsteps
        calls of step()."""
        import torch
        from .particles import FIELDS
        pg, s = self.pgroup, self.solver
        n = pg.np
        if self.sort_interval:
            raise ValueError("run_host: the host owns the particle order; use sort_interval=0")
        main = torch.cuda.current_stream(pg.device)
        if not hasattr(self, "_h2d"):
            self._h2d = torch.cuda.Stream(pg.device)
            self._d2h = torch.cuda.Stream(pg.device)
        h2d, d2h = self._h2d, self._d2h
        edges = [n * k // nchunks for k in range(nchunks + 1)]
        landed = [None] * nchunks
        brought = [None] * nchunks  # chunk k is back on the host

        def upload():
            for k in range(nchunks):
                if brought[k] is None:
                    h2d.wait_stream(main)
                else:
                    h2d.wait_event(brought[k])
                a, b = edges[k], edges[k + 1]
                with torch.cuda.stream(h2d):
                    for f in FIELDS:
                        getattr(pg, f)[a:b].copy_(host[f][a:b], non_blocking=True)
                ev = torch.cuda.Event()
                ev.record(h2d)
                landed[k] = ev

        upload()
        for it in range(nsteps):
            center = self._center()
            s.deposit_begin()
            for k in range(nchunks):
                a, b = edges[k], edges[k + 1]
                main.wait_event(landed[k])
                if b > a:
                    s.advance(pg, self.dt, prwall=self.cfg["pipe_radius"], start=a, stop=b, center=center,
                              deposit=True)
                ev = torch.cuda.Event()
                ev.record(main)
                d2h.wait_event(ev)
                with torch.cuda.stream(d2h):
                    for f in FIELDS:
                        host[f][a:b].copy_(getattr(pg, f)[a:b], non_blocking=True)
                back = torch.cuda.Event()
                back.record(d2h)
                brought[k] = back
            s.deposit_end(zero_first=True)
            self.vsync = False
            if it + 1 < nsteps:
                upload()
            if self.warmstart is not None:
                self.warmstart.guess(s)
            s.solve()
            self.it += 1
        main.wait_stream(d2h)

    def synchv(self, nzmmnt=0, zmmntmin=None, zmmntmax=None):
        """padvnc3d("synchv") at the end of a special step (w3d.F:975): a
        half kick with the field of the last solve takes the velocities from
        t - dt/2 to t, where the positions are. The next step is then halfv.
        Does nothing when the velocities are already in step.

        With nzmmnt > 0 it also takes the moments of that step, as the
        synchv call of getzmmnt does (w3d.F:2327-2345): the moments on a z
        grid of nzmmnt cells over [zmmntmin, zmmntmax) (default the field
        grid) with each particle extrapolated in time using its velocity
        change over the half step, and the global moments. The moments
        (diagnostics.finalize, keys as the reference's pnum, xrms, epsx,
        pnumz, xrmsz, epsxz, ...) are appended to self.history with the step
        number and time, and returned."""
        if self.vsync:
            return None
        pg = self.pgroup
        uold = (pg.ux.clone(), pg.uy.clone(), pg.uz.clone()) if nzmmnt > 0 else None
        self.solver.advance(pg, self.dt, prwall=self.cfg["pipe_radius"], center="synchv")
        self.vsync = True
        if not nzmmnt:
            return None
        from .diagnostics import finalize
        zmin = self.cfg["zmmin"] if zmmntmin is None else zmmntmin
        zmax = self.cfg["zmmax"] if zmmntmax is None else zmmntmax
        z0, zm = self.solver.zmoments(pg, uold, 0.5 * self.dt, zmin, zmax, nzmmnt)
        out = {"it": self.it, "time": self.it * self.dt}
        out.update(finalize(z0))
        out.update(finalize(zm, "z"))
        if not hasattr(self, "history"):
            self.history = []
        self.history.append(out)
        return out

    def moments(self):
        """Moments of the particles as they are; call synchv() first for
        velocities at the positions' time (the reference's special step)."""
        return self.solver.moments(self.pgroup)

    def dump(self, filename=None, prefix="", runid="espic", suffix=""):
        """Restartable dump of the run (the dump/restart pair of
        scripts/warp.py:950-1121, as one .npz file): the workload, the solver
        options, the step counter, the particle arrays and phi with its guard
        cells. rho is not saved: every step deposits it afresh. The default
        name follows the reference's prefix + runid + '%06d' % it + suffix +
        '.dump'. Returns the file name."""
        import json
        if filename is None:
            filename = "%s%s%06d%s.dump.npz" % (prefix, runid, self.it, suffix)
        s, pg = self.solver, self.pgroup
        arrays = {"p_" + k: v for k, v in pg.to_numpy().items()}
        meta = {"cfg": self.cfg, "it": self.it, "vsync": self.vsync, "sort_interval": self.sort_interval,
                "precision": s.precision, "particle_dtype": "float32" if pg.fp32 else "float64",
                "tolkind": s.tolkind, "mgtol": s.mgtol, "mgmaxiters": s.mgmaxiters, "q": pg.q, "m": pg.m,
                "w": pg.w}
        with open(filename, "wb") as f:
            np.savez(f, meta=np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8),
                     phi=s.phi.cpu().numpy(), **arrays)
        return filename


def restart(filename, device="cuda"):
    """Rebuilds an ESPIC run from ESPIC.dump: same workload, options, step
    counter, particles and phi, so the following steps reproduce the run
    that wrote the dump bit for bit."""
    import json
    with np.load(filename) as d:
        meta = json.loads(bytes(d["meta"]).decode())
        parts = {k[2:]: d[k] for k in d.files if k.startswith("p_")}
        phi = d["phi"]
    import torch
    run = ESPIC(meta["cfg"], precision=meta["precision"], tolkind=meta["tolkind"], mgtol=meta["mgtol"],
                mgmaxiters=meta["mgmaxiters"], device=device, particles=parts, sort_interval=meta["sort_interval"],
                particle_dtype=getattr(torch, meta.get("particle_dtype", "float64")))
    run.pgroup.q, run.pgroup.m, run.pgroup.w = meta["q"], meta["m"], meta["w"]
    run.solver.phi = np.asfortranarray(phi)
    run.it = meta["it"]
    run.vsync = meta["vsync"]
    return run
