"""Training and evaluation of the learned multigrid warm start.

Snapshots come from the plain solver running randomized beams on one of the
synthetic workloads (by default the 128x128x256-cell grid over the
8 cm x 8 cm x 1 m box). The beam parameters are drawn as follows:
- current uniform in 1-50 mA;
- emittance log-uniform in 1-20 mm mrad;
- envelope mismatch uniform in 0-30 %.

Each snapshot is one PIC step, taken after the deposit. Its inputs are the
residual field of phi^(n-1) under rho^n and phi^(n-1) itself. Its target is
phi^n from the FP64 multigrid solved to a 1e-8 relative residual. The network
is trained on the GPU with the library's tensor-core convolutions (forward,
data and weight gradients) and Adam; 10 % of the snapshots are held out.

The evaluation runs fresh beams. At every step it solves to a 1e-6 relative
residual twice from the same rho^n: once warm-started from phi^(n-1) (the
plain method), and once from phi^(n-1) plus the network's correction. It
reports the V-cycles of both, and the relative residual right after each
start.

    python -m warp_b200.warmstart_train --snapshots 400 --epochs 6 --out ws.pt
"""
import argparse
import json
import math
import time

import numpy as np
import torch

from . import pic
from .particles import semigaussian_device
from .unet import UNet3D, WarmStart, check_errors


def beam_params(rng):
    current = rng.uniform(1e-3, 50e-3)
    emit = math.exp(rng.uniform(math.log(1.0), math.log(20.0))) * 1e-6  # m rad
    mismatch = rng.uniform(0.0, 0.30)
    return current, emit, mismatch


def beam_run(workload, rng, gen, device, npart=None, mgtol=1e-6, sort_interval=4, precision="mixed"):
    """A run of one randomized beam, with its initial field solved (by
    default as the learned form runs: mixed precision to a 1e-6 relative
    residual)."""
    current, emit, mismatch = beam_params(rng)
    cfg = pic.workload(workload, current=current, mismatch=mismatch, angle_rms=emit / (2 * 4e-3),
                       seed=int(rng.integers(1 << 30)))
    if npart:
        cfg["npart"] = npart
    beam = semigaussian_device(cfg["npart"], gen, radius=cfg["radius"], mismatch=mismatch,
                               angle_rms=cfg["angle_rms"], device=device)
    run = pic.ESPIC(cfg, precision=precision, tolkind="relres", mgtol=mgtol, device=device, particles=beam,
                    sort_interval=sort_interval)
    run.generate()
    return run, {"current": current, "emittance": emit, "mismatch": mismatch}


def snapshots(n, workload="D", seed=0, device="cuda", steps_per_beam=8, skip=2, npart=None, log=print,
              factor=1):
    """Returns (inputs [n] of [D,H,W,2] bf16, residual scales s_r [n],
    masked scaled corrections m (phi^n - phi^(n-1)) / s_r [n] of [D,H,W]
    bf16, meta, the mask m of the network grid). The runs solve as the
    learned form does (mixed precision, 1e-6 relative residual), so the
    inputs are those the network meets in use. factor: the network's grid is
    the workload's coarsened that many times. Stored in bf16 on the device:
    25 MB a snapshot on the 128x128x256 grid at factor 1. Every beam of a
    workload has the same conductors, hence one mask."""
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device).manual_seed(seed)
    ws = WarmStart(None, factor=factor)
    xs, srs, zs, meta = [], [], [], []
    mask = None
    t0 = time.time()
    while len(xs) < n:
        run, m = beam_run(workload, rng, gen, device, npart)
        s = run.solver
        for k in range(skip + steps_per_beam):
            s.advance(run.pgroup, run.dt, prwall=run.cfg["pipe_radius"])
            s.loadrho()
            if k >= skip and len(xs) < n:
                x, s_r = ws.inputs(s)
                phi_prev = s.phi.clone()
                s.solve()
                zs.append(ws.target(s, phi_prev, s_r))
                xs.append(x)
                srs.append(s_r)
                meta.append(dict(m, step=k))
                if mask is None:
                    mask = ws._net_mask(s).clone()
                del phi_prev
            else:
                s.solve()
        run.close()
        del run
    log("snapshots: %d in %.1f s" % (len(xs), time.time() - t0))
    return xs, srs, zs, meta, mask


def fit_out_scale(srs, zs):
    """Median over snapshots of rms(phi^n - phi^(n-1)) / s_r."""
    return float(np.median([float(torch.sqrt(torch.mean(z.float() ** 2)).item()) for z in zs]))


def targets(srs, zs, out_scale):
    """Training targets (phi^n - phi^(n-1)) / (s_r * out_scale), bf16."""
    return [(z.float() * (1.0 / out_scale)).to(torch.bfloat16).contiguous() for z in zs]


def _pad16(x2):
    x = torch.zeros(x2.shape[:3] + (16,), dtype=torch.bfloat16, device=x2.device)
    x[..., :2] = x2
    return x


def laplacian(u):
    """7-point Laplacian (grid units) of [D,H,W] u on the interior nodes."""
    c = u[1:-1, 1:-1, 1:-1]
    return (u[:-2, 1:-1, 1:-1] + u[2:, 1:-1, 1:-1] + u[1:-1, :-2, 1:-1] + u[1:-1, 2:, 1:-1] + u[1:-1, 1:-1, :-2] +
            u[1:-1, 1:-1, 2:] - 6. * c)


def guess_loss(pred, y, lap_weight, mask=None):
    """MSE of the correction plus lap_weight times the MSE of its Laplacian:
    the multigrid measures a guess by its residual, which the Laplacian of the
    error dominates, so high-frequency error costs more than its size. The
    prediction counts on the unmasked nodes only (the guess adds nothing
    elsewhere)."""
    if mask is not None:
        pred = pred * mask
    e = pred - y.float()
    return torch.mean(e * e) + lap_weight * torch.mean(laplacian(e) ** 2)


def train(xs, ys, epochs=6, lr=1e-3, seed=0, device="cuda", lap_weight=1.0, clip=1.0, log=print, mask=None):
    """Adam over the snapshots in a seeded order, the gradient norm clipped
    to `clip` (without it a first large step can silence the ReLUs of a
    layer, and the network then outputs a constant). The gradients come from
    the library's kernels, summed in a fixed order, so a training is the same
    bits on every run."""
    net = UNet3D(seed=seed, device=device)
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    n = len(xs)
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        t0 = time.time()
        tot = 0.0
        for i in rng.permutation(n):
            pred = net(_pad16(xs[i]))
            loss = guess_loss(pred, ys[i], lap_weight, mask)
            opt.zero_grad(set_to_none=True)
            loss.backward()
            torch.nn.utils.clip_grad_norm_(net.parameters(), clip)
            opt.step()
            tot += float(loss.item())
        check_errors(torch.device(device))
        for g in opt.param_groups:
            g["lr"] *= 0.7
        hist.append(tot / n)
        log("epoch %d: train mse %.4e (%.1f s)" % (ep, tot / n, time.time() - t0))
    return net, hist


@torch.no_grad()
def evaluate(net, xs, ys, mask=None):
    """Held-out MSE of the network and of the zero prediction (the plain
    warm start phi^(n-1)), on the unmasked nodes when a mask is given."""
    m, m0 = 0.0, 0.0
    for x2, y in zip(xs, ys):
        p = net(_pad16(x2))
        if mask is not None:
            p = p * mask
        m += float(torch.mean((p - y.float()) ** 2))
        m0 += float(torch.mean(y.float() ** 2))
    return m / len(xs), m0 / len(xs)


@torch.no_grad()
def vcycle_study(ws, workload="D", nbeams=2, steps=6, seed=1000, device="cuda", npart=None, precision="mixed",
                 mgtol=1e-6, guard=False):
    """V-cycles to mgtol from the plain warm start and from the learned
    guess, on the same rho^n, over fresh randomized beams (guard: the
    guess is taken back where it is the worse start, WarmStart.guess)."""
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device).manual_seed(seed)
    rows = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(nbeams):
        run, _m = beam_run(workload, rng, gen, device, npart, mgtol=mgtol, precision=precision)
        s = run.solver
        for k in range(steps):
            s.advance(run.pgroup, run.dt, prwall=run.cfg["pipe_radius"])
            s.loadrho()
            phi_prev = s.phi.clone()
            r_plain = s.relresidual()
            s.solve()
            n_plain = s.mgiters
            s.phi.copy_(phi_prev)
            e0.record()
            ws.guess(s, guard=guard)
            e1.record()
            torch.cuda.synchronize()
            r_learned = s.relresidual()
            s.solve()
            rows.append({"step": k, "vc_plain": n_plain, "vc_learned": s.mgiters, "relres_start_plain": r_plain,
                         "relres_start_learned": r_learned, "guess_ms": e0.elapsed_time(e1)})
        run.close()
        del run
    vp = float(np.mean([r["vc_plain"] for r in rows]))
    vl = float(np.mean([r["vc_learned"] for r in rows]))
    return {"vcycles_plain": vp, "vcycles_learned": vl,
            "relres_start_plain": float(np.median([r["relres_start_plain"] for r in rows])),
            "relres_start_learned": float(np.median([r["relres_start_learned"] for r in rows])),
            "guess_ms": float(np.median([r["guess_ms"] for r in rows])), "steps": len(rows)}


def main():
    """Generates the snapshots, trains, and studies the V-cycles on fresh beams
    of the training workload (the network on its grid coarsened by
    --factor) and, with --study-b, of the 256x256x512 workload (coarsened by
    twice that, the same cell size). Writes the weights to --out and the
    results (JSON) to --json."""
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="D")
    ap.add_argument("--snapshots", type=int, default=400)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--npart", type=int, default=None)
    ap.add_argument("--out", default="warmstart_weights.pt")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--study-beams", type=int, default=2)
    ap.add_argument("--study-steps", type=int, default=6)
    ap.add_argument("--lap-weight", type=float, default=1.0)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--study-b", action="store_true")
    ap.add_argument("--factor", type=int, default=1, choices=[1, 2, 4],
                    help="the network's grid is the workload's coarsened this many times")
    ap.add_argument("--json", default=None)
    args = ap.parse_args()
    torch.cuda.set_device(0)
    xs, srs, zs, meta, mask = snapshots(args.snapshots, workload=args.workload, seed=args.seed, npart=args.npart,
                                        factor=args.factor)
    out_scale = fit_out_scale(srs, zs)
    ys = targets(srs, zs, out_scale)
    del zs
    nval = max(1, len(xs) // 10)
    t0 = time.time()
    net, hist = train(xs[nval:], ys[nval:], epochs=args.epochs, seed=args.seed, lap_weight=args.lap_weight,
                      mask=mask)
    train_s = time.time() - t0
    mse, mse0 = evaluate(net, xs[:nval], ys[:nval], mask)
    study = {}
    for sm in WarmStart.SMOOTH:
        ws = WarmStart(net, out_scale=out_scale, smooth=sm, factor=args.factor)
        study[sm] = vcycle_study(ws, workload=args.workload, nbeams=args.study_beams, steps=args.study_steps,
                                 npart=args.npart, precision=args.precision)
    best = min(study, key=lambda k: study[k]["vcycles_learned"])
    ws = WarmStart(net, out_scale=out_scale, smooth=best, factor=args.factor)
    ws.train_factor = args.factor
    torch.save(ws.state(), args.out)
    res = {"workload": args.workload, "factor": args.factor, "snapshots": len(xs), "heldout": nval,
           "epochs": args.epochs,
           "lap_weight": args.lap_weight, "out_scale": out_scale, "train_s": train_s, "heldout_mse": mse,
           "heldout_mse_zero_guess": mse0, "ratio": mse / mse0, "train": hist, "study": study, "smooth": best}
    if args.study_b:
        del xs, ys
        torch.cuda.empty_cache()
        wsb = WarmStart(net, out_scale=out_scale, smooth=best, factor=2 * args.factor)
        res["study_B"] = vcycle_study(wsb, workload="B", nbeams=1, steps=args.study_steps, precision=args.precision)
    print(json.dumps(res))
    if args.json:
        with open(args.json, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
