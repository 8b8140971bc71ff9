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
    xs, srs, ds, _ = wt.snapshots(64, workload="A", seed=5, log=lambda *a: None)
    out_scale = wt.fit_out_scale(srs, ds)
    ys = wt.targets(srs, ds, out_scale)
    nval = 8
    net, hist = wt.train(xs[nval:], ys[nval:], epochs=4, seed=5, log=lambda *a: None)
    mse, mse0 = wt.evaluate(net, xs[:nval], ys[:nval])
    print("held-out mse: learned %.4g, zero correction %.4g (ratio %.3f)" % (mse, mse0, mse / mse0))
    # a second training from the same seed gives the same weights
    net2, _ = wt.train(xs[nval:nval + 8], ys[nval:nval + 8], epochs=1, seed=5, log=lambda *a: None)
    net3, _ = wt.train(xs[nval:nval + 8], ys[nval:nval + 8], epochs=1, seed=5, log=lambda *a: None)
    for k, v in net2.state_dict().items():
        assert torch.equal(v, net3.state_dict()[k]), k
    assert hist[-1] < hist[0]
    assert mse < 0.8 * mse0
    ws = WarmStart(net, out_scale=out_scale, smooth="coarse4")
    st = wt.vcycle_study(ws, workload="A", nbeams=1, steps=4, seed=77, precision="fp64")
    print("V-cycles to 1e-6: plain %.2f, learned %.2f; start relres plain %.3g, learned %.3g; guess %.2f ms" % (
        st["vcycles_plain"], st["vcycles_learned"], st["relres_start_plain"], st["relres_start_learned"],
        st["guess_ms"]))
    # every learned-start solve converged (mgmaxiters is 100)
    assert st["vcycles_learned"] < 100
    assert st["vcycles_plain"] < 100
