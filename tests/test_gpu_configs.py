"""The benchmark configurations at full size, checked through properties
that do not need a CPU reference run at that size. At these sizes the CPU
oracle takes minutes per solve; the bit-level parity with it is checked at
the smaller sizes in the other test files.

- C: standalone solve on a 512^3 grid. rho is 64 random Gaussian blobs; the
  conductors are a grounded cylinder and 8 spheres at random potentials.
  FP64 and mixed precision are both solved to a 1e-10 relative residual.
  Checks: both converge, conductor interior nodes hold their voltage
  exactly, and the two solutions agree.
- B: the 256x256x512 grid with 5e7 particles, two PIC steps in each form.
  Checks: the deposited charge equals the particles' charge, each solve
  reaches 1e-6, the pipe holds 0 V, and the forms agree.
- E: the 256x256x1024 grid with 2e8 particles and four quadrupole rods at
  +-20 kV. Checks: the rods hold their voltage exactly, the solve converges,
  and charge is conserved.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _blobs_rho(solver, nblob, seed, eps0):
    from warp_b200.workloads import blobs_rho
    blobs_rho(solver, nblob, seed, eps0 * 1e4)


def _interior_check(solver):
    """Finest-level interior conductor nodes hold their voltage exactly."""
    ii, iv, il = solver.conductor_data()["interior"]
    sel = il == 0
    idx = torch.as_tensor(ii[sel].astype(np.int64) + 1, device=solver.device)
    got = solver.phi[idx[:, 0], idx[:, 1], idx[:, 2]].cpu().numpy()
    assert sel.sum() > 0
    assert np.array_equal(got, iv[sel])


def test_config_C_512cubed_fp64_and_mixed():
    from warp_b200.constants import eps0
    from warp_b200.multigrid import MultiGridB200
    torch.cuda.set_device(0)
    from warp_b200.workloads import config_c_shapes
    shapes = config_c_shapes()
    phis, iters = {}, {}
    for prec in ("fp64", "mixed"):
        s = MultiGridB200(512, 512, 512, 0., 1., 0., 1., 0., 1., bounds=(0, 0, 0, 0, 0, 0), mgtol=1e-10,
                          tolkind="relres", mgmaxiters=200, precision=prec)
        for sh in shapes:
            s.installconductor(sh)
        _blobs_rho(s, 64, 7, eps0)
        s.solve()
        assert s.converged and s.relres <= 1e-10
        _interior_check(s)
        phis[prec] = s.phi.clone()
        iters[prec] = s.mgiters
        del s
        torch.cuda.empty_cache()
    scale = float(phis["fp64"].abs().max())
    diff = float((phis["fp64"] - phis["mixed"]).abs().max())
    print("C 512^3: V-cycles fp64 %d, mixed %d; max|phi| %.3g V, max diff %.3g V" % (
        iters["fp64"], iters["mixed"], scale, diff))
    assert scale > 0.1
    assert diff <= 1e-7 * scale


def _run(workload, precision, steps, npart=None):
    from warp_b200 import pic
    from warp_b200.particles import semigaussian_device
    cfg = pic.workload(workload)
    if npart:
        cfg["npart"] = npart
    gen = torch.Generator(device="cuda").manual_seed(11)
    beam = semigaussian_device(cfg["npart"], gen, radius=cfg["radius"], mismatch=cfg["mismatch"],
                               angle_rms=cfg["angle_rms"])
    run = pic.ESPIC(cfg, precision=precision, tolkind="relres", mgtol=1e-6, particles=beam, sort_interval=10)
    run.generate()
    for _ in range(steps):
        run.step()
        assert run.solver.converged and run.solver.relres <= 1e-6
    return run


def _charge_check(run):
    s, pg = run.solver, run.pgroup
    s.loadrho(lfinalize_rho=False)
    total = float(s.rho.sum()) * s.dx * s.dy * s.dz
    expect = pg.nlive() * pg.q * pg.w
    assert abs(total - expect) <= 1e-12 * abs(expect)


def test_config_B_full_size_two_steps():
    torch.cuda.set_device(0)
    runs = {}
    for prec in ("fp64", "mixed"):
        r = _run("B", prec, 2)
        _interior_check(r.solver)
        runs[prec] = (r.solver.phi.clone(), r.moments())
        _charge_check(r)
        del r
        torch.cuda.empty_cache()
    (pa, ma), (pb, mb) = runs["fp64"], runs["mixed"]
    scale = float(pa.abs().max())
    diff = float((pa - pb).abs().max())
    print("B: max|phi| %.4g V, fp64 - mixed %.3g V; epsx %.6g / %.6g" % (scale, diff, ma["epsx"], mb["epsx"]))
    assert diff <= 1e-3 * scale
    assert ma["n"] == mb["n"]
    assert abs(ma["epsx"] - mb["epsx"]) <= 1e-5 * ma["epsx"]


def test_config_E_full_size_rods():
    torch.cuda.set_device(0)
    r = _run("E", "mixed", 1)
    _interior_check(r.solver)
    ii, iv, il = r.solver.conductor_data()["interior"]
    assert set(np.unique(iv[il == 0]).tolist()) >= {20e3, -20e3}
    _charge_check(r)
