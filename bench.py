#!/usr/bin/env python
"""Benchmark of the 3D electrostatic PIC step on B200.

Workload: 256x256x512 cells over 8 cm x 8 cm x 1 m, 5e7 protons at 1 MeV
(semi-Gaussian, 4 mm radius, 20% envelope mismatch, 5 mrad, 10 mA), FODO of
hard-edge quads (10 cm, +-15 T/m, 50 cm period), grounded pipe r = 3.5 cm,
periodic z; seeded synthetic beam. One step = fused gather+push+boundaries,
fixed-point deposition, multigrid solve to a 1e-6 relative residual (warm
started from the previous phi).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Prints one JSON line (rank 0). Under torchrun each rank runs an independent
replica (the path does not shard; "replicas only") and the timing is the
max over ranks.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PIC steps/s, 256²×512 grid/5e7 ptcl: plain vs learned+mixed @1e-6 residual"
WORKLOAD = "B"
# particles are re-sorted by cell every SORT_INTERVAL steps (inside the timed steps)
SORT_INTERVAL = 10
# DRAM bytes (read + write) per finest-level node of one launch, from ncu
# captures of one launch on the 257x257x513-node level: k_sor_bulk<float>
# (one half sweep, bulk nodes and the colour's subgrid points): 311.2 MB read
# + 94.6 MB written.
TRAFFIC_PER_NODE = {"k_sor_bulk<float>": (311.19488e6 + 94.622976e6) / (257 * 257 * 513)}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--forms", default="plain,mixed,learned")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-steps", type=int, default=2,
                    help="oracle steps timed for cpu_baseline (continuing the GPU run's state)")
    ap.add_argument("--npart", type=int, default=None, help="override the particle count (profiling runs)")
    return ap.parse_args()


def max_over_ranks(ms, world, device):
    """Slowest rank's time (device-timed per rank): every replica ran the
    same number of steps, so the job took as long as the slowest one."""
    if world <= 1:
        return ms
    import torch
    import torch.distributed as tdist
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(ms_per_step, world):
    """Whole-job steps/s of `world` independent replicas."""
    return world * 1000.0 / ms_per_step


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.proc.terminate()
        self.proc.wait()
        rows = [l.split(",") for l in open(self.path).read().strip().splitlines() if l.strip()]
        os.unlink(self.path)
        sm = sorted(float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit())
        smax = max((float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()),
                   default=None)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for k, n in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(rows)}


WEIGHTS = os.path.join(ROOT, "warp_b200", "weights", "warmstart_D.pt")


def load_warmstart(dev):
    """The committed network, trained on the 128x128x256 workload coarsened
    by train_factor, run on the 256x256x512 (and 256x256x1024) grids
    coarsened by twice that, so that it sees the cell size it was trained
    at."""
    import torch

    from warp_b200.unet import WarmStart
    st = torch.load(WEIGHTS, map_location="cpu")
    return WarmStart.load(st, device=dev, factor=2 * int(st.get("train_factor", 1)))


class TimedGuess:
    """The learned guess with CUDA-event timing of every call."""

    def __init__(self, ws):
        self.ws = ws
        self.events = []
        self.results = []  # (relres of phi^(n-1), relres of the guess, kept)

    def guess(self, solver):
        import torch
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        self.results.append(self.ws.guess(solver))
        b.record()
        self.events.append((a, b))

    def summary(self):
        """Of the steps: the fraction where the network ran, and where its
        guess was kept; the median starting residuals of the runs."""
        r = self.results
        if not r:
            return {}
        ran = [x for x in r if x[0] is not None]
        med = lambda v: sorted(v)[len(v) // 2] if v else None
        return {"guess_ran_fraction": len(ran) / len(r), "guess_kept_fraction": sum(1 for x in r if x[2]) / len(r),
                "relres_start_plain_median": med([x[0] for x in ran]),
                "relres_start_learned_median": med([x[1] for x in ran])}

    def ms(self):
        """Duration of each guess() call that ran the network."""
        import torch
        torch.cuda.synchronize()
        return [a.elapsed_time(b) for (a, b), x in zip(self.events, self.results) if x[0] is not None]


def run_form(name, cfg, beam, steps, warmup, dev, prof):
    """One form of the step: plain (FP64 throughout), mixed (FP32 V-cycles in
    FP64 defect correction, FP32 particles and push) or learned (mixed with
    the learned initial guess before every solve: the U-Net trained on the
    128x128x256 workload, applied on this grid coarsened by two)."""
    import torch

    from warp_b200 import _lib
    from warp_b200.pic import ESPIC
    precision = {"plain": "fp64", "mixed": "mixed", "learned": "mixed"}[name]
    run = ESPIC(cfg, precision=precision, tolkind="relres", mgtol=1e-6, device=dev, particles=beam,
                sort_interval=SORT_INTERVAL)
    timed = None
    if name == "learned":
        timed = TimedGuess(load_warmstart(dev))
    run.generate()
    s = run.solver
    run.warmstart = timed
    run.step(warmup)
    # one untimed re-sort: the first sort of a process loads and sizes the
    # sort's kernels and buffers, which would otherwise fall into the timed
    # steps of whichever form runs first
    run.pgroup.sort(s)
    if timed is not None:
        timed.events.clear()
        timed.results.clear()
    stream = torch.cuda.current_stream()
    h = s._h
    n0 = _lib.ctypes.c_int64()
    _lib.check(_lib.lib.wg_launch_count(h, _lib.ctypes.byref(n0)))
    vc = 0
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        run.step()
        vc += s.mgiters
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    n1 = _lib.ctypes.c_int64()
    _lib.check(_lib.lib.wg_launch_count(h, _lib.ctypes.byref(n1)))
    out = {"ms_per_step": ms / steps, "vcycles_per_solve": vc / steps, "launches": n1.value - n0.value,
           "live": run.pgroup.nlive(), "relres": s.relres}
    if timed is not None:
        g = timed.ms()
        out["guess_ms"] = sum(g) / len(g) if g else None
        out.update(timed.summary())
        out["weights"] = os.path.relpath(WEIGHTS, ROOT)
    if prof:
        # kernel durations from CUDA events on the launching stream, over the
        # same number of further steps (event timing runs the V-cycles kernel
        # by kernel instead of from the captured graph)
        kinds = {"sor0": _lib.PROF_SOR0, "advance": _lib.PROF_ADVANCE,
                 "deposit": _lib.PROF_DEPOSIT, "resid0": _lib.PROF_RESID0, "restrict0": _lib.PROF_RESTRICT0,
                 "expand0": _lib.PROF_EXPAND0, "corr": _lib.PROF_CORR, "coarse": _lib.PROF_COARSE}
        mask = 0
        for v in kinds.values():
            mask |= 1 << v
        _lib.check(_lib.lib.wg_prof_enable(h, mask))
        for _ in range(steps):
            run.step()
        out["kernels"] = {}
        for k, v in kinds.items():
            t, n, u = _lib.ctypes.c_double(), _lib.ctypes.c_int64(), _lib.ctypes.c_double()
            _lib.check(_lib.lib.wg_prof_read(h, v, _lib.ctypes.byref(t), _lib.ctypes.byref(n), _lib.ctypes.byref(u)))
            out["kernels"][k] = {"ms": t.value, "launches": n.value, "units": u.value}
        _lib.check(_lib.lib.wg_prof_enable(h, 0))
    return run, out


def e2e_steps(run, steps):
    """The drop-in path with host-owned particles (WARP's pgroup lives in
    host memory): every step moves the 7 particle arrays host->device from
    pinned memory and back through ESPIC.run_host, which pipelines the
    copies in chunks against the advance and the deposit, and queues the
    next step's uploads before the field solve."""
    import torch
    from warp_b200.particles import FIELDS
    pg = run.pgroup
    # the host owns the particle order in this mode: no device-side re-sort
    run.sort_interval = 0
    host = {k: torch.empty(pg.np, dtype=pg.dtype, pin_memory=True) for k in FIELDS}
    for k in FIELDS:
        host[k].copy_(getattr(pg, k))
    run.step_host(host)  # warm-up (creates the copy streams)
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    run.run_host(host, steps)
    e1.record(stream)
    torch.cuda.synchronize()
    nbytes = sum(host[k].numel() * host[k].element_size() for k in FIELDS)
    return e0.elapsed_time(e1) / steps, nbytes, nbytes


def oracle_steps(orun, warmup, steps):
    """Times `steps` full PIC steps of the oracle run after `warmup` untimed
    ones; returns (seconds per step, V-cycles per solve)."""
    for _ in range(warmup):
        orun.step()
    vc, t = 0, 0.0
    for _ in range(steps):
        t0 = time.perf_counter()
        vc += orun.step()
        t += time.perf_counter() - t0
    return t / max(steps, 1), vc / max(steps, 1)


def oracle_desc(cfg, threads, steps, npart, start):
    return ("oracle (C++ FP64 restatement of the reference's Fortran, %d host threads): %d full PIC steps "
            "(gather+push, deposit and multigrid to 1e-6 relative residual) of %d particles on the %dx%dx%d "
            "grid, %s" % (threads, steps, npart, cfg["nx"], cfg["ny"], cfg["nz"], start))


def job_config(cfg, world):
    """The config object of the JSON line, identical in both arms."""
    n = cfg["npart"]
    e = len(str(n)) - len(str(n).rstrip("0"))
    npart = "%de%d" % (n // 10 ** e, e) if e >= 3 else str(n)
    return {"workload": "%dx%dx%d cells, %s protons, pipe%s + FODO, 1e-6 relres"
                        % (cfg["nx"], cfg["ny"], cfg["nz"], npart, " + 4 rods" if cfg.get("rods") else ""),
            "parallelism": "replicas" if world > 1 else "single",
            "flush": "inputs larger than L2 (phi %d MB, particles %.1f GB)"
                     % (8 * (cfg["nx"] + 3) * (cfg["ny"] + 3) * (cfg["nz"] + 3) // 10 ** 6, 56e-9 * n)}


def reference_arm(args, cfg, world):
    """The reference's arithmetic on the host cores: the oracle's PIC steps
    on the same workload, nothing of the CUDA library loaded."""
    from oracle import oracle
    from oracle.espic import OracleESPIC
    orun = OracleESPIC(cfg, tolkind="relres", mgtol=1e-6)
    orun.generate()
    sec, vc = oracle_steps(orun, args.warmup, args.steps)
    threads = oracle.threads()
    v = 1.0 / sec
    desc = oracle_desc(cfg, threads, args.steps, len(orun.p["x"]),
                       "after %d untimed steps from the loaded beam" % args.warmup)
    return {"metric": METRIC, "value": v, "unit": "steps/s", "impl": "reference", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded semi-Gaussian beam)",
            "config": job_config(cfg, world), "form": "reference arithmetic (FP64 oracle on the host cores)",
            "vcycles_per_solve": vc,
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": threads, "kind": "port", "sample": desc},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def config_c(args, dev):
    """Config C: the standalone multigrid solve on the 512^3 grid (64 Gaussian
    blobs, grounded cylinder and 8 spheres at seeded potentials) to a 1e-10
    relative residual from phi = 0, FP64 and mixed. Reports solve time,
    V-cycles and the finest-level smoother's HBM GB/s (per-launch CUDA
    events). One JSON line; `value` is the mixed form's solves/s."""
    import torch

    from warp_b200 import _lib
    from warp_b200.constants import eps0
    from warp_b200.multigrid import MultiGridB200
    from warp_b200.workloads import CONFIG_C, blobs_rho, config_c_shapes
    n = CONFIG_C["n"]
    peak, peak_kind = measured_peaks()
    forms = {}
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    for prec in ("fp64", "mixed"):
        s = MultiGridB200(n, n, n, 0., 1., 0., 1., 0., 1., bounds=(0, 0, 0, 0, 0, 0), mgtol=CONFIG_C["mgtol"],
                          tolkind="relres", mgmaxiters=200, precision=prec, mgverbose=-1, device=dev)
        for sh in config_c_shapes():
            s.installconductor(sh)
        blobs_rho(s, CONFIG_C["nblob"], CONFIG_C["blob_seed"], eps0 * 1e4)
        s.solve()  # conductor set-up and graph capture
        ms = []
        for _ in range(max(args.steps, 1)):
            s.phi.zero_()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            s.solve()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        assert s.converged
        vc, rr = s.mgiters, s.relres
        s.phi.zero_()
        _lib.check(_lib.lib.wg_prof_enable(s._h, 1 << _lib.PROF_SOR0))
        s.solve()
        t, c, u = _lib.ctypes.c_double(), _lib.ctypes.c_int64(), _lib.ctypes.c_double()
        _lib.check(_lib.lib.wg_prof_read(s._h, _lib.PROF_SOR0, _lib.ctypes.byref(t), _lib.ctypes.byref(c),
                                         _lib.ctypes.byref(u)))
        _lib.check(_lib.lib.wg_prof_enable(s._h, 0))
        t, c, u = t.value, c.value, u.value
        bpn = 6.0 if prec == "mixed" else 12.0
        gbs = bpn * u / (t * 1e-3) / 1e9 if c else None
        forms[prec] = {"ms_per_solve": sum(ms) / len(ms), "vcycles": vc, "relres": rr,
                       "smoother": {"kernel": "k_sor_bulk" + ("<float>" if prec == "mixed" else "<double>") +
                                    " (finest level, one red or black half sweep)",
                                    "launches": c, "us_per_launch": 1e3 * t / c if c else None,
                                    "bytes_per_node_per_launch": bpn, "achieved_gbs": gbs,
                                    "frac": gbs / peak if gbs else None}}
        del s
        torch.cuda.empty_cache()
    clk = clocks.stop()
    return {"metric": "multigrid solve, 512^3 grid, cylinder + 8 spheres, 64 blobs, to 1e-10 relres",
            "value": 1000.0 / forms["mixed"]["ms_per_solve"], "unit": "solves/s", "n_gpus": 1,
            "steps": max(args.steps, 1), "higher_is_better": True, "dtype": "f32+f64",
            "data": "synthetic (seeded Gaussian blobs)", "config": {"workload": "C: 512x512x512 cells"},
            "forms": forms, "peak": peak, "peak_kind": peak_kind, "clocks": clk}


def config_e(args, dev):
    """Config E: the combined run on the 256x256x1024 grid with 2e8 particles,
    the FODO lattice and four electrostatic quadrupole rods (+-20 kV) inside
    the grounded pipe. The combined form (learned guess + FP32 multigrid in
    FP64 defect correction + FP32 push, fixed-point deposit) runs against the
    plain FP64 form from the same seeded beam for args.steps steps. Every
    `every` steps both bring their velocities to the positions' time
    (synchv, the reference's special step) and record the emittances, the
    live count and the field energy (getese3dfromrhophi). One JSON line:
    ms/step and V-cycles of each form, the records, and the largest
    relative differences of the combined form from the plain one."""
    import torch

    from warp_b200.particles import semigaussian_device
    from warp_b200.pic import ESPIC
    from warp_b200.workloads import workload
    cfg = workload("E")
    every = max(1, min(50, args.steps))
    forms, recs = {}, {}
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    for name in ("plain", "combined"):
        gen = torch.Generator(device=dev).manual_seed(cfg["seed"])
        beam = semigaussian_device(cfg["npart"], gen, radius=cfg["radius"], mismatch=cfg["mismatch"],
                                   angle_rms=cfg["angle_rms"], zmin=cfg["zmmin"], zmax=cfg["zmmax"],
                                   ekin_ev=cfg["ekin_ev"], device=dev)
        run = ESPIC(cfg, precision="fp64" if name == "plain" else "mixed", tolkind="relres", mgtol=1e-6,
                    device=dev, particles=beam, sort_interval=SORT_INTERVAL)
        del beam
        timed = None
        if name == "combined" and os.path.exists(WEIGHTS):
            timed = TimedGuess(load_warmstart(dev))
            run.warmstart = timed
        run.generate()
        rows, ms, vc, nsolve = [], 0.0, 0, 0
        done = 0
        while done < args.steps:
            k = min(every, args.steps - done)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(k):
                run.step()
                vc += run.solver.mgiters
                nsolve += 1
            e1.record()
            torch.cuda.synchronize()
            ms += e0.elapsed_time(e1)
            done += k
            run.synchv()
            m = run.moments()
            rows.append({"it": run.it, "n": m["n"], "epsx": m["epsx"], "epsy": m["epsy"], "xrms": m["xrms"],
                         "ese": run.solver.getese()})
        out = {"ms_per_step": ms / args.steps, "vcycles_per_solve": vc / max(nsolve, 1)}
        if timed is not None:
            g = timed.ms()
            out["guess_ms"] = sum(g) / len(g) if g else None if g else None
            out.update(timed.summary())
        forms[name], recs[name] = out, rows
        run.close()
        del run
        torch.cuda.empty_cache()
    clk = clocks.stop()
    diff = {}
    for key in ("epsx", "epsy", "xrms", "ese"):
        d = [abs(c[key] - p[key]) / abs(p[key]) for p, c in zip(recs["plain"], recs["combined"]) if p[key]]
        diff[key] = {"max_rel": max(d) if d else None, "final_rel": d[-1] if d else None}
    diff["n"] = {"final_plain": recs["plain"][-1]["n"], "final_combined": recs["combined"][-1]["n"]}
    return {"metric": "combined form vs plain FP64, 256x256x1024 grid, 2e8 particles, FODO + 4 rods",
            "value": 1000.0 / forms["combined"]["ms_per_step"], "unit": "steps/s", "n_gpus": 1,
            "steps": args.steps, "higher_is_better": True, "dtype": "f32+f64",
            "data": "synthetic (seeded semi-Gaussian beam)", "config": {"workload": "E: 256x256x1024 cells, 2e8 "
                                                                        "protons, pipe + 4 rods + FODO"},
            "forms": forms, "records_every": every, "records": recs, "combined_vs_plain": diff, "clocks": clk}


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.workload == "C":
        import torch
        torch.cuda.set_device(local)
        if rank == 0:
            print(json.dumps(config_c(args, "cuda:%d" % local)))
        return 0
    if args.workload == "E" and args.impl != "reference":
        import torch
        torch.cuda.set_device(local)
        if rank == 0:
            print(json.dumps(config_e(args, "cuda:%d" % local)))
        return 0
    from warp_b200.workloads import workload
    cfg = workload(args.workload) if args.npart is None else workload(args.workload, npart=args.npart)
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(reference_arm(args, cfg, world)))
        return 0

    import torch
    import torch.distributed as tdist
    from datetime import timedelta
    torch.cuda.set_device(local)
    dev = "cuda:%d" % local
    if world > 1:
        tdist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device(dev))
    from warp_b200.particles import semigaussian
    beam = semigaussian(cfg["npart"], seed=cfg["seed"] + rank, radius=cfg["radius"], mismatch=cfg["mismatch"],
                        angle_rms=cfg["angle_rms"], zmin=cfg["zmmin"], zmax=cfg["zmmax"], ekin_ev=cfg["ekin_ev"])
    forms = [f for f in args.forms.split(",") if f]
    skipped = {}
    if "learned" in forms and not os.path.exists(WEIGHTS):
        forms.remove("learned")
        skipped["learned"] = "no trained weights at %s" % os.path.relpath(WEIGHTS, ROOT)
    headline = forms[-1]
    results = {}
    clocks = None
    head_run = None
    for f in forms:
        prof = f == headline
        if world > 1:
            tdist.barrier()
        if prof:
            clocks = Clocks(local)
            clocks.start()
        run, res = run_form(f, cfg, beam, args.steps, args.warmup, dev, prof)
        if prof:
            clk = clocks.stop()
            head_run = run
        else:
            run.close()
            del run
            torch.cuda.empty_cache()
        results[f] = res
    ms_head = max_over_ranks(results[headline]["ms_per_step"], world, dev)
    value = replica_throughput(ms_head, world)
    e2e_ms, h2d, d2h = e2e_steps(head_run, args.e2e_steps) if args.e2e_steps > 0 else (float("nan"), 0, 0)
    e2e_ms = max_over_ranks(e2e_ms, world, dev)
    peak, peak_kind = measured_peaks()
    kern = results[headline]["kernels"]
    fp32 = headline != "plain"
    # The dominant level-0 smoother launch, one red or black half sweep, and
    # its algorithmic bytes per node: the hot-path table counts 24 B/node for
    # a full red+black sweep in FP64 and 12 B/node in FP32, so a half sweep
    # moves 12 and 6.
    sor = kern["sor0"]
    bytes_per_node = 6.0 if fp32 else 12.0
    sor_kernel = "k_sor_bulk<%s> (finest level, one red or black half sweep)" % ("float" if fp32 else "double")
    achieved = None
    if sor["launches"]:
        per_launch_bytes = bytes_per_node * sor["units"] / sor["launches"]
        achieved = per_launch_bytes / (sor["ms"] / sor["launches"] * 1e-3) / 1e9
    tpn = TRAFFIC_PER_NODE.get(sor_kernel.split(" ")[0])
    roofline = {"bound": "hbm", "kernel": sor_kernel, "achieved": achieved,
                "peak": peak, "unit": "GB/s", "frac": (achieved / peak) if achieved else None,
                "peak_kind": peak_kind,
                "traffic": (tpn * sor["units"] / sor["launches"] if tpn and sor["launches"] else None),
                "bytes_per_node_per_launch": bytes_per_node}
    ratios = {}
    if "plain" in results:
        p = results["plain"]
        for f in ("mixed", "learned"):
            if f in results:
                ratios["steps_per_s_%s_over_plain" % f] = p["ms_per_step"] / results[f]["ms_per_step"]
                ratios["vcycles_plain_over_%s" % f] = p["vcycles_per_solve"] / results[f]["vcycles_per_solve"]
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_head, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if headline == "plain" else "f32+f64",
            "data": "synthetic (seeded semi-Gaussian beam)",
            "config": job_config(cfg, world), "form": headline,
            "forms": results, "ratios": ratios, "gpu_launches": results[headline]["launches"],
            "e2e": {"value": 1000.0 / e2e_ms * world, "unit": "steps/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": roofline, "clocks": clk}
    if skipped:
        line["skipped_forms"] = skipped
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.cpu_steps > 0:
        # the oracle continues the GPU run from its current particles and
        # phi for a few full steps (a bounded sample of the same workload)
        from oracle import oracle
        from oracle.espic import OracleESPIC
        pg = head_run.pgroup
        orun = OracleESPIC(cfg, particles=pg.to_numpy(), w=pg.w, phi=head_run.solver.phi.cpu().numpy(),
                           vsync=head_run.vsync)
        sec, vc = oracle_steps(orun, 0, args.cpu_steps)
        line["cpu_baseline"] = {"value": 1.0 / sec, "unit": "steps/s", "cores": oracle.threads(), "kind": "port",
                                "sample": oracle_desc(cfg, oracle.threads(), args.cpu_steps, len(orun.p["x"]),
                                                      "continuing the GPU run's particles and phi"),
                                "vcycles_per_solve": vc}
        del orun
    if world > 1:
        tdist.barrier()
        tdist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
