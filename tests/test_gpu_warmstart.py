"""The learned warm start, trained on the GPU with the library's tensor-core
convolutions, against the method without it (the previous step's phi).

The network is trained on snapshots of the plain solver on the
32x32x64-cell workload with randomized beams. The test checks two things:
- On held-out snapshots, the network's correction is closer to the true
  phi^n - phi^(n-1) than the zero correction of the plain warm start.
- Multigrid still converges to the 1e-6 relative residual from the
  learned guess; the plain solver still decides when each step has converged.

The V-cycle counts of both starts are measured and printed. On this problem
the learned start saves no V-cycles, and the test records that rather than
asserting a gain.

The weight gradients are summed in a fixed order, so a training is the same
bits on every run: one seed, no retry.
"""
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_learned_warm_start_gain_and_convergence():
    from warp_b200 import warmstart_train as wt
    from warp_b200.unet import WarmStart
    torch.cuda.set_device(0)
    xs, srs, ds, _, mask = wt.snapshots(64, workload="A", seed=5, log=lambda *a: None)
    out_scale = wt.fit_out_scale(srs, ds)
    ys = wt.targets(srs, ds, out_scale)
    nval = 8
    net, hist = wt.train(xs[nval:], ys[nval:], epochs=4, seed=5, log=lambda *a: None, mask=mask)
    mse, mse0 = wt.evaluate(net, xs[:nval], ys[:nval], mask)
    print("held-out mse: learned %.4g, zero correction %.4g (ratio %.3f)" % (mse, mse0, mse / mse0))
    # a second training from the same seed gives the same weights
    net2, _ = wt.train(xs[nval:nval + 8], ys[nval:nval + 8], epochs=1, seed=5, log=lambda *a: None)
    net3, _ = wt.train(xs[nval:nval + 8], ys[nval:nval + 8], epochs=1, seed=5, log=lambda *a: None)
    for k, v in net2.state_dict().items():
        assert torch.equal(v, net3.state_dict()[k]), k
    assert hist[-1] < hist[0]
    assert mse < 0.8 * mse0
    ws = WarmStart(net, out_scale=out_scale, smooth="none")
    st = wt.vcycle_study(ws, workload="A", nbeams=1, steps=4, seed=77)
    print("V-cycles to 1e-6: plain %.2f, learned %.2f; start relres plain %.3g, learned %.3g; guess %.2f ms" % (
        st["vcycles_plain"], st["vcycles_learned"], st["relres_start_plain"], st["relres_start_learned"],
        st["guess_ms"]))
    # every learned-start solve converged (mgmaxiters is 100)
    assert st["vcycles_learned"] < 100
    assert st["vcycles_plain"] < 100


def test_committed_weights_on_a_heldout_beam():
    """The committed weights (trained on 4000 snapshots of the 128x128x256
    workload) on a beam drawn from a seed the training did not use.

    - From the second step on, the predicted change of phi matches the true
      change on the unmasked nodes (farther than the margin from every
      conductor): its mean squared error is below 10 % of the zero guess's
      (the plain warm start phi^(n-1)).
    - The guard keeps a guess only when it starts MIN_GAIN times lower than
      phi^(n-1); a rejected guess restores phi^(n-1) bit for bit.
    - Every solve from the guess reaches the 1e-6 relative residual.
    - Over the steps after the first, the solves from the guess take fewer
      V-cycles in total than those from phi^(n-1) (the plain warm start,
      f3d_mgrid.F:313-317).
    The starting residuals and V-cycles of both starts are printed."""
    import os
    import numpy as np
    from warp_b200 import warmstart_train as wt
    from warp_b200.unet import WarmStart
    torch.cuda.set_device(0)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    ws = WarmStart.load(os.path.join(root, "warp_b200", "weights", "warmstart_D.pt"), device="cuda")
    ws.backoff = 1  # the network on every step, whatever the guard decided before
    rng = np.random.default_rng(4242)
    gen = torch.Generator(device="cuda").manual_seed(4242)
    run, _ = wt.beam_run("D", rng, gen, "cuda")
    s = run.solver
    core = WarmStart._core_phi
    rows = []
    for k in range(4):
        s.advance(run.pgroup, run.dt, prwall=run.cfg["pipe_radius"])
        s.loadrho()
        phi_prev = s.phi.clone()
        xin, s_r = ws.inputs(s)
        m = ws.node_mask(s)
        pred = ws.predict(xin) * (s_r * ws.out_scale) * m
        s.solve()
        n_plain = s.mgiters
        d = (core(s.phi) - core(phi_prev)) * m
        ratio = float((pred - d).pow(2).sum() / d.pow(2).sum())
        s.phi.copy_(phi_prev)
        r_plain, r_guess, kept = ws.guess(s)
        if kept:
            assert r_guess * ws.MIN_GAIN <= r_plain
        else:
            assert torch.equal(s.phi, phi_prev)
        s.solve()
        assert s.converged and s.relres <= 1e-6
        rows.append((k, ratio, r_plain, r_guess, kept, n_plain, s.mgiters))
        print("step %d: mse ratio %.4f, relres start plain %.3g learned %.3g (%s), V-cycles plain %d learned %d" % (
            k, ratio, r_plain, r_guess, "kept" if kept else "rejected", n_plain, s.mgiters))
    run.close()
    assert all(r[1] < 0.1 for r in rows[1:]), rows
    assert sum(r[6] for r in rows[1:]) < sum(r[5] for r in rows[1:]), rows
