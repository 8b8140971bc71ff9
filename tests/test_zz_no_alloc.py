"""wg_deposit_noalloc: the deposit for callers that cannot let a library
allocate device memory (a host code that manages every device buffer
itself, or one that keeps cudaMalloc/cudaFree, which synchronize the device,
out of its step). Its fixed-point accumulator is a fixed array inside the
library, so it takes no context and allocates nothing.

Checked through the C ABI against the context deposit wg_deposit on the same
particles, two calls in a row (clear, then accumulate): both run the same
fixed-point kernels with the same cell sizes, so the results must agree bit
for bit. The first call is also checked against the oracle's FP64 running
sum, device memory must not change across the calls, and grids above the
limit are rejected. Collected last (file name) so that it also runs after
every other test."""
import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle

pytestmark = pytest.mark.gpu

MAX_NODES = 1 << 20


def _grid(cfg, bounds=(0, 0, 0, 0, 2, 2)):
    from warp_b200 import _lib
    g = _lib.Grid()
    g.nx, g.ny, g.nz = cfg["nx"], cfg["ny"], cfg["nz"]
    g.xmmin, g.xmmax, g.ymmin, g.ymmax = cfg["xmmin"], cfg["xmmax"], cfg["ymmin"], cfg["ymmax"]
    g.zmmin, g.zmmax = cfg["zmmin"], cfg["zmmax"]
    for k in range(6):
        g.bounds[k] = bounds[k]
    return g


def _noalloc(grid, pg, rho, zero_first):
    from warp_b200 import _lib
    s = pg.cstruct()
    stream = torch.cuda.current_stream(pg.device).cuda_stream
    return _lib.lib.wg_deposit_noalloc(ctypes.byref(grid), ctypes.byref(s), ctypes.c_void_p(rho.data_ptr()),
                                       int(zero_first), ctypes.c_void_p(stream))


def test_noalloc_deposit_matches_context_deposit_twice():
    from warp_b200 import _lib, pic
    from warp_b200.multigrid import MultiGridB200
    from warp_b200.particles import ParticleGroup, semigaussian
    torch.cuda.set_device(0)
    cfg = pic.workload("A")
    s = MultiGridB200(cfg["nx"], cfg["ny"], cfg["nz"], cfg["xmmin"], cfg["xmmax"], cfg["ymmin"], cfg["ymmax"],
                      cfg["zmmin"], cfg["zmmax"], bounds=(0, 0, 0, 0, 2, 2), mgverbose=-1)
    p1 = semigaussian(200_000, seed=11, radius=4e-3, mismatch=0.2)
    p1["gaminv"][::89] = 0.0
    p2 = semigaussian(150_000, seed=12, radius=3e-3)
    g1, g2 = ParticleGroup(p1, w=1e4), ParticleGroup(p2, w=2.5e4)
    grid = _grid(cfg)
    nr = (cfg["nx"] + 1) * (cfg["ny"] + 1) * (cfg["nz"] + 1)
    rho = torch.full((nr,), 7.0, dtype=torch.float64, device=g1.device)  # garbage that zero_first must replace

    # first call: rho = deposit(p1)
    _lib.check(_noalloc(grid, g1, rho, 1))
    torch.cuda.synchronize()
    a1 = rho.cpu().numpy().copy()
    s.loadrho(pgroups=[g1], lfinalize_rho=False)
    torch.cuda.synchronize()
    r1 = s.rho.cpu().numpy().ravel(order="F")
    assert np.array_equal(a1, r1)
    # and against the oracle's FP64 running sum (the fixed-point rounding of
    # each weight to 2^-46 is the only difference)
    ref = np.zeros((cfg["nx"] + 1, cfg["ny"] + 1, cfg["nz"] + 1), order="F")
    oracle.setrho(ref, p1["x"], p1["y"], p1["z"], g1.q, g1.w, s.dx, s.dy, s.dz, s.xmmin, s.ymmin, s.zmmin,
                  gaminv=p1["gaminv"])
    ref = ref.ravel(order="F")
    scale = np.max(np.abs(ref))
    assert scale > 0
    assert np.max(np.abs(a1 - ref)) <= 1e-13 * scale

    # second call right after: rho += deposit(p2); the accumulator must have
    # been cleared, and nothing is allocated on the device
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    _lib.check(_noalloc(grid, g2, rho, 0))
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    a2 = rho.cpu().numpy()
    _lib.check(_lib.lib.wg_deposit(s._h, ctypes.byref(g2.cstruct()), 0))
    torch.cuda.synchronize()
    r2 = s.rho.cpu().numpy().ravel(order="F")
    assert np.array_equal(a2, r2)
    assert not np.array_equal(a2, a1)


def test_noalloc_deposit_rejects_grids_above_the_limit():
    from warp_b200 import _lib
    from warp_b200.particles import ParticleGroup, semigaussian
    torch.cuda.set_device(0)
    pg = ParticleGroup(semigaussian(1000, seed=1), w=1.0)
    cfg = dict(nx=128, ny=128, nz=64, xmmin=-0.04, xmmax=0.04, ymmin=-0.04, ymmax=0.04, zmmin=0.0, zmmax=1.0)
    assert 129 * 129 * 65 > MAX_NODES
    rho = torch.zeros(1, dtype=torch.float64, device=pg.device)
    rc = _noalloc(_grid(cfg), pg, rho, 1)
    assert rc == -7  # WG_ETOOLARGE
    assert b"fixed limit of 1048576 nodes" in _lib.lib.wg_last_error()
