"""Training of the learned multigrid warm start on snapshots of the plain
solver (workload D: 128x128x256 cells over the 8 cm x 8 cm x 1 m box).

Each snapshot is one PIC step of a randomized beam -- current uniform in
1-50 mA, emittance log-uniform in 1-20 mm mrad, envelope mismatch uniform
in 0-30 % -- taken after the deposit: inputs rho^n and phi^(n-1), target
phi^n from the FP64 multigrid solved to a 1e-8 relative residual. The
network is trained on the GPU with the library's tensor-core convolutions
(forward, data and weight gradients) and Adam; 10 % of the snapshots are
held out.

    python -m warp_b200.warmstart_train --snapshots 400 --epochs 8 --out w.pt
"""
import argparse
import json
import math
import time

import numpy as np
import torch

from . import pic
from .constants import eps0
from .particles import semigaussian_device
from .unet import UNet3D, WarmStart, check_errors


def beam_params(rng):
    current = rng.uniform(1e-3, 50e-3)
    emit = math.exp(rng.uniform(math.log(1.0), math.log(20.0))) * 1e-6  # m rad
    mismatch = rng.uniform(0.0, 0.30)
    return current, emit, mismatch


def make_warmstart(net, cfg):
    dx = (cfg["xmmax"] - cfg["xmmin"]) / cfg["nx"]
    return WarmStart(net, rho_factor=10.0 * dx * dx / eps0, out_scale=30.0)


def snapshots(n, seed=0, device="cuda", steps_per_beam=4, skip=2, npart=None, log=print):
    """Returns (inputs [n] of [D,H,W,2] bf16, targets [n] of [D,H,W] bf16,
    meta list)."""
    rng = np.random.default_rng(seed)
    gen = torch.Generator(device=device).manual_seed(seed)
    xs, ys, meta = [], [], []
    t0 = time.time()
    while len(xs) < n:
        current, emit, mismatch = beam_params(rng)
        cfg = pic.workload("D", current=current, mismatch=mismatch, angle_rms=emit / (2 * 4e-3),
                           seed=int(rng.integers(1 << 30)))
        if npart:
            cfg["npart"] = npart
        beam = semigaussian_device(cfg["npart"], gen, radius=cfg["radius"], mismatch=mismatch,
                                   angle_rms=cfg["angle_rms"], device=device)
        run = pic.ESPIC(cfg, tolkind="relres", mgtol=1e-8, device=device, particles=beam, sort_interval=4)
        ws = make_warmstart(None, cfg)
        run.generate()
        s = run.solver
        for k in range(skip + steps_per_beam):
            s.advance(run.pgroup, run.dt, prwall=cfg["pipe_radius"])
            s.loadrho()
            phi_prev = s.phi.clone()
            s.solve()
            if k >= skip and len(xs) < n:
                x, y = ws.pair(s.rho, phi_prev, s.phi)
                xs.append(x)
                ys.append(y)
                meta.append({"current": current, "emittance": emit, "mismatch": mismatch, "step": k})
        del run
    log("snapshots: %d in %.1f s" % (len(xs), time.time() - t0))
    return xs, ys, meta


def train(xs, ys, epochs=8, lr=2e-3, seed=0, device="cuda", log=print):
    net = UNet3D(seed=seed, device=device)
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    n = len(xs)
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        t0 = time.time()
        tot = 0.0
        for i in rng.permutation(n):
            x = torch.zeros(xs[i].shape[:3] + (16,), dtype=torch.bfloat16, device=device)
            x[..., :2] = xs[i]
            pred = net(x)
            loss = torch.mean((pred - ys[i].float()) ** 2)
            opt.zero_grad(set_to_none=True)
            loss.backward()
            opt.step()
            tot += float(loss.item())
        check_errors(torch.device(device))
        for g in opt.param_groups:
            g["lr"] *= 0.7
        hist.append(tot / n)
        log("epoch %d: train mse %.4e (%.1f s)" % (ep, tot / n, time.time() - t0))
    return net, hist


@torch.no_grad()
def evaluate(net, xs, ys, device="cuda"):
    """Held-out MSE of the network and of the zero prediction (the plain
    warm start phi^(n-1))."""
    m, m0 = 0.0, 0.0
    for x2, y in zip(xs, ys):
        x = torch.zeros(x2.shape[:3] + (16,), dtype=torch.bfloat16, device=device)
        x[..., :2] = x2
        p = net(x)
        m += float(torch.mean((p - y.float()) ** 2))
        m0 += float(torch.mean(y.float() ** 2))
    return m / len(xs), m0 / len(xs)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--snapshots", type=int, default=400)
    ap.add_argument("--epochs", type=int, default=8)
    ap.add_argument("--npart", type=int, default=None)
    ap.add_argument("--out", default="warmstart_weights.pt")
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    torch.cuda.set_device(0)
    xs, ys, meta = snapshots(args.snapshots, seed=args.seed, npart=args.npart)
    nval = max(1, len(xs) // 10)
    net, hist = train(xs[nval:], ys[nval:], epochs=args.epochs, seed=args.seed)
    mse, mse0 = evaluate(net, xs[:nval], ys[:nval])
    print(json.dumps({"heldout_mse": mse, "heldout_mse_zero_guess": mse0, "ratio": mse / mse0, "train": hist}))
    torch.save({k: v.detach().cpu() for k, v in net.state_dict().items()}, args.out)


if __name__ == "__main__":
    main()
