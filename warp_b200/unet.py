"""Learned multigrid warm start: a small 3D U-Net that predicts phi^n from
(rho^n, phi^(n-1)); multigrid always finishes the solve from that guess.

The 3x3x3 convolutions (forward, data gradient, weight gradient) run on the
library's BF16 tcgen05 kernels with FP32 accumulation (wg_conv3_fwd,
wg_conv3_wgrad). PyTorch provides the autograd graph, the 2x average pooling,
nearest-neighbour upsampling, concatenation, the loss and the Adam
optimiser -- the training glue.

Tensors are channels-last [D][H][W][C] (z, y, x) in bf16 on the device, for
one sample at a time. Architecture (4 levels, 16/32/64/128 channels):
  enc1 conv 16->16, 16->16 | pool | enc2 16->32, 32->32 | pool |
  enc3 32->64, 64->64 | pool | mid 64->128, 128->128 | up, cat enc3 |
  dec3 192->64, 64->64 | up, cat enc2 | dec2 96->32, 32->32 | up, cat enc1 |
  dec1 48->16, 16->16 | out 16->16 (channel 0 is the prediction)
ReLU after every convolution except the last. The two inputs are padded to
16 channels with zeros.
"""
import ctypes
import math

import torch

from . import _lib

_ERR = {}


def _errbuf(device):
    b = _ERR.get(device)
    if b is None:
        b = _ERR[device] = torch.zeros(1, dtype=torch.int32, device=device)
    return b


def check_errors(device):
    """Raises if a convolution kernel reported a timed-out wait."""
    b = _errbuf(device)
    if int(b.item()) != 0:
        b.zero_()
        raise RuntimeError("tensor-core convolution: an mbarrier wait timed out")


def _stream(device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def pack_weights(w):
    """[27, Cout, Cin] -> [27, Cin/8, Cout, 8]: the layout wg_conv3_fwd reads,
    in which the weights of one tap and one block of input channels are
    contiguous."""
    t, cout, cin = w.shape
    return w.view(t, cout, cin // 8, 8).permute(0, 2, 1, 3).contiguous()


def conv3_fwd(x, w, bias=None, relu=False, out=None, yoff=0, mask=None, out_dtype=torch.bfloat16):
    """x: [D,H,W,Cin] bf16; w: [27,Cout,Cin] bf16; bias fp32 [Cout] or None.
    Writes channels yoff..yoff+Cout-1 of `out` ([D,H,W,Ctot], bf16, or FP32
    with out_dtype=torch.float32: the accumulator without the bf16
    rounding)."""
    D, H, W, cin = x.shape
    cout = w.shape[1]
    assert x.dtype == torch.bfloat16 and w.dtype == torch.bfloat16 and x.is_contiguous() and w.is_contiguous()
    assert w.shape == (27, cout, cin)
    wp = pack_weights(w)
    if out is None:
        out = torch.empty((D, H, W, cout), dtype=out_dtype, device=x.device)
    assert out.is_contiguous() and out.shape[:3] == (D, H, W) and out.dtype in (torch.bfloat16, torch.float32)
    if mask is not None:
        assert mask.is_contiguous() and mask.shape[:3] == (D, H, W)
    err = _errbuf(x.device)
    fn = _lib.lib.wg_conv3_fwd_f32 if out.dtype == torch.float32 else _lib.lib.wg_conv3_fwd
    _lib.check(fn(
        x.data_ptr(), D, H, W, cin, wp.data_ptr(), bias.data_ptr() if bias is not None else None, cout,
        out.data_ptr(), out.shape[3], yoff, mask.data_ptr() if mask is not None else None,
        mask.shape[3] if mask is not None else 0, int(relu), err.data_ptr(), _stream(x.device)))
    return out


_SCRATCH = {}


def _wgrad_scratch(cin, cout, device):
    """Partial-sum scratch of wg_conv3_wgrad, kept per (device, cin, cout)."""
    key = (device, cin, cout)
    t = _SCRATCH.get(key)
    if t is None:
        n = ctypes.c_int64()
        _lib.check(_lib.lib.wg_conv3_wgrad_scratch(cin, cout, ctypes.byref(n)))
        t = _SCRATCH[key] = torch.empty(n.value, dtype=torch.float32, device=device)
    return t


def conv3_wgrad(x, dy):
    """dW[t][co][ci] = sum_v dy[v][co] x[v+off_t][ci] (fp32), deterministic."""
    D, H, W, cin = x.shape
    cout = dy.shape[3]
    assert x.is_contiguous() and dy.is_contiguous()
    dw = torch.empty((27, cout, cin), dtype=torch.float32, device=x.device)
    scratch = _wgrad_scratch(cin, cout, x.device)
    err = _errbuf(x.device)
    _lib.check(_lib.lib.wg_conv3_wgrad(x.data_ptr(), dy.data_ptr(), D, H, W, cin, cout, dw.data_ptr(),
                                       scratch.data_ptr(), scratch.numel(), err.data_ptr(), _stream(x.device)))
    return dw


def flip_transpose(w):
    """Weights of the data-gradient convolution: w'[t][ci][co] = w[26-t][co][ci]."""
    return w.flip(0).transpose(1, 2).contiguous()


class _Conv3(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, w, b, relu, f32):
        wb = w.to(torch.bfloat16).contiguous()
        y = conv3_fwd(x.contiguous(), wb, b.float().contiguous(), relu=relu,
                      out_dtype=torch.float32 if f32 else torch.bfloat16)
        ctx.save_for_backward(x, wb, y)
        ctx.relu = relu
        return y

    @staticmethod
    def backward(ctx, gy):
        x, wb, y = ctx.saved_tensors
        g = gy.to(torch.bfloat16)
        if ctx.relu:
            g = g * (y > 0)
        g = g.contiguous()
        dx = conv3_fwd(g, flip_transpose(wb), None, relu=False)
        dw = conv3_wgrad(x.contiguous(), g)
        db = g.float().sum(dim=(0, 1, 2))
        return dx, dw, db, None, None


def conv3(x, w, b, relu=True, f32=False):
    """The convolution as an autograd op; f32: FP32 output (the gradient
    still flows in bf16)."""
    return _Conv3.apply(x, w, b, relu, f32)


def _pool(x):
    D, H, W, C = x.shape
    return x.view(D // 2, 2, H // 2, 2, W // 2, 2, C).float().mean(dim=(1, 3, 5)).to(torch.bfloat16)


def _up(x):
    return x.repeat_interleave(2, 0).repeat_interleave(2, 1).repeat_interleave(2, 2)


LAYERS = [("e1a", 16, 16), ("e1b", 16, 16), ("e2a", 16, 32), ("e2b", 32, 32), ("e3a", 32, 64), ("e3b", 64, 64),
          ("m1", 64, 128), ("m2", 128, 128), ("d3a", 192, 64), ("d3b", 64, 64), ("d2a", 96, 32), ("d2b", 32, 32),
          ("d1a", 48, 16), ("d1b", 16, 16), ("out", 16, 16)]


class UNet3D(torch.nn.Module):
    def __init__(self, seed=0, device="cuda"):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.w = torch.nn.ParameterDict()
        self.b = torch.nn.ParameterDict()
        for name, cin, cout in LAYERS:
            std = math.sqrt(2.0 / (27 * cin)) * (0.1 if name == "out" else 1.0)
            self.w[name] = torch.nn.Parameter((torch.randn(27, cout, cin, generator=g) * std).to(device))
            self.b[name] = torch.nn.Parameter(torch.zeros(cout, device=device))

    def c(self, name, x, relu=True, f32=False):
        return conv3(x, self.w[name], self.b[name], relu, f32)

    def forward(self, x):
        """x: [D,H,W,16] bf16 (2 used channels); returns [D,H,W] FP32 (the
        last layer's accumulator, not rounded to bf16)."""
        e1 = self.c("e1b", self.c("e1a", x))
        e2 = self.c("e2b", self.c("e2a", _pool(e1)))
        e3 = self.c("e3b", self.c("e3a", _pool(e2)))
        m = self.c("m2", self.c("m1", _pool(e3)))
        d3 = self.c("d3b", self.c("d3a", torch.cat([_up(m), e3], dim=3)))
        d2 = self.c("d2b", self.c("d2a", torch.cat([_up(d3), e2], dim=3)))
        d1 = self.c("d1b", self.c("d1a", torch.cat([_up(d2), e1], dim=3)))
        # the prediction in FP32: rounding it to bf16 would add noise whose
        # Laplacian is a residual of its own
        return self.c("out", d1, relu=False, f32=True)[..., 0].contiguous()


class WarmStart:
    """The learned guess around the solver's arrays. For a step n the network
    sees, on the nodes 0..nx-1, 0..ny-1, 0..nz-1 (z, y, x order):
      channel 0: m * r / s_r, with r = rhs(rho^n) - A phi^(n-1) the residual
                 field of the previous potential under the new charge
                 (MultiGridB200.residual_field), m the conductor mask below
                 and s_r the rms of m * r over the unmasked nodes;
      channel 1: phi^(n-1) / s_p, with s_p the rms of phi^(n-1).
    Both are functions of (rho^n, phi^(n-1)) only. It predicts
    (phi^n - phi^(n-1)) / (s_r * out_scale) on the unmasked nodes, which is
    O(1) because the correction is the residual passed through the inverse
    Laplacian; out_scale is fixed from the training snapshots.

    The mask m is 0 within `margin` cells of a conductor node of the finest
    level and on Dirichlet boundary planes, 1 elsewhere. Next to a subgrid
    conductor the stored residual is the unscaled row of the conductor
    stencil, which grows as the inverse of the boundary distance; left in,
    those few nodes set s_r and swamp the beam. And a correction next to a
    conductor is the error the V-cycles remove slowest, so the guess leaves
    those nodes at phi^(n-1)."""

    # Low-pass filters applied to the prediction before it is added: the
    # multigrid measures a guess by its residual, and the bf16 output carries
    # rounding and fitting noise whose Laplacian is as large as the residual
    # it removes. "box2": two passes of a 3x3x3 mean; "coarse4": mean over
    # 4x4x4 blocks, then trilinear interpolation back.
    SMOOTH = ("none", "box2", "coarse4")

    def __init__(self, net, out_scale=1.0, smooth="none", factor=1, margin=2, out_margin=6, backoff=10):
        """factor 1: the network runs on the solver's grid (nodes 0..n-1 per
        axis). factor f = 2 or 4: it runs on that grid coarsened f times in
        each direction -- the inputs are means over f^3 node blocks, and the
        predicted correction is interpolated back trilinearly (cell-centred,
        the transfer pair of avg_pool3d and interpolate(align_corners=False))
        -- so a network trained at one cell size serves a grid f times finer
        than its training grid coarsened by f.
        margin: cells around conductor nodes where the inputs are zeroed (as
        in training); out_margin: cells around them where the guess changes
        nothing (corrections there are the error the V-cycles reduce
        slowest: measured on the 128x128x256 workload, a 6-cell margin took
        the solves from the guess from 5-7 to 4 V-cycles).
        backoff: after the guard rejects a guess, the next backoff - 1 calls
        of guess() return at once (phi^(n-1) stays the start) and the one
        after tries the network again; 1 tries it on every call."""
        if smooth not in self.SMOOTH:
            raise ValueError("smooth must be one of %s" % (self.SMOOTH,))
        if factor not in (1, 2, 4):
            raise ValueError("factor must be 1, 2 or 4")
        self.net = net
        self.out_scale = float(out_scale)
        self.smooth = smooth
        self.factor = factor
        self.margin = int(margin)
        self.out_margin = int(out_margin)
        self.backoff = max(1, int(backoff))
        self._skip = 0
        self.calls = 0   # guess() calls
        self.tried = 0   # of them, those that ran the network
        self._rbuf = None
        self._masks = {}

    def lowpass(self, d):
        """d: [D,H,W] float32 prediction -> filtered copy."""
        if self.smooth == "none":
            return d
        u = d[None, None]
        if self.smooth == "box2":
            for _ in range(2):
                u = torch.nn.functional.avg_pool3d(u, 3, stride=1, padding=1, count_include_pad=False)
        else:
            c = torch.nn.functional.avg_pool3d(u, 4, stride=4)
            u = torch.nn.functional.interpolate(c, size=d.shape, mode="trilinear", align_corners=False)
        return u[0, 0]

    @staticmethod
    def _core_phi(phi):
        return phi[1:-2, 1:-2, 1:-2].permute(2, 1, 0)

    def _coarsen(self, u):
        """[D,H,W] on the solver's nodes -> the network's grid."""
        if self.factor == 1:
            return u
        return torch.nn.functional.avg_pool3d(u[None, None], self.factor)[0, 0]

    def node_mask(self, solver, margin=None):
        """The mask m ([D,H,W] float32 on the solver's nodes 0..n-1) for
        `margin` cells (default the input margin), built from the finest
        level's conductor nodes and kept until the conductor counts
        change."""
        import numpy as np
        margin = self.margin if margin is None else int(margin)
        solver.getconductorobject()
        counts = np.zeros(3, np.int64)
        _lib.check(_lib.lib.wg_conductors_counts(solver._h, counts.ctypes.data_as(_lib._i64p)))
        key = (id(solver), tuple(int(c) for c in counts), solver.nx, solver.ny, solver.nz, tuple(solver.bounds))
        hit = self._masks.get(margin)
        if hit is not None and hit[0] == key:
            return hit[1]
        nx, ny, nz = solver.nx, solver.ny, solver.nz
        cd = solver.conductor_data()
        pts = [cd["interior"][0][cd["interior"][2] == 0], cd["subgrid"][0][cd["subgrid"][3] == 0]]
        idx = np.concatenate(pts).astype(np.int64) if sum(len(p) for p in pts) else np.zeros((0, 3), np.int64)
        ok = (idx >= 0).all(axis=1) & (idx[:, 0] < nx) & (idx[:, 1] < ny) & (idx[:, 2] < nz)
        idx = torch.as_tensor(idx[ok], device=solver.device)
        g = torch.zeros((nz, ny, nx), dtype=torch.float32, device=solver.device)
        if len(idx):
            g[idx[:, 2], idx[:, 1], idx[:, 0]] = 1.0
        if margin > 0:
            g = torch.nn.functional.max_pool3d(g[None, None], 2 * margin + 1, stride=1, padding=margin)[0, 0]
        m = 1.0 - g
        b = solver.bounds
        if b[0] == 0:
            m[:, :, 0] = 0.
        if b[2] == 0:
            m[:, 0, :] = 0.
        if b[4] == 0:
            m[0, :, :] = 0.
        m = m.contiguous()
        self._masks[margin] = (key, m)
        return m

    def _net_mask(self, solver):
        """The input mask on the network's grid: a coarse node counts when
        all of its fine nodes do."""
        m = self.node_mask(solver)
        if self.factor == 1:
            return m
        return -torch.nn.functional.max_pool3d(-m[None, None], self.factor)[0, 0]

    def inputs(self, solver):
        """([D,H,W,2] bf16 inputs, s_r) from the solver's rho and phi (phi
        holds phi^(n-1)), on the network's grid."""
        n = (solver.nx + 1) * (solver.ny + 1) * (solver.nz + 1)
        if self._rbuf is None or self._rbuf.numel() != n or self._rbuf.device != solver.device:
            self._rbuf = torch.empty(n, dtype=torch.float64, device=solver.device)
        m = self._net_mask(solver)
        r = self._coarsen(solver.residual_field(out=self._rbuf)[:-1, :-1, :-1].permute(2, 1, 0)) * m
        p = self._coarsen(self._core_phi(solver.phi))
        cnt = float(m.sum().item()) or 1.0
        s_r = float(torch.sqrt(torch.sum(r * r) / cnt).item()) or 1.0
        s_p = float(torch.sqrt(torch.mean(p * p)).item()) or 1.0
        x = torch.empty(r.shape + (2,), dtype=torch.bfloat16, device=r.device)
        x[..., 0] = (r * (1.0 / s_r)).to(torch.bfloat16)
        x[..., 1] = (p * (1.0 / s_p)).to(torch.bfloat16)
        return x.contiguous(), s_r

    def target(self, solver, phi_prev, s_r):
        """Training target of one solved step (solver.phi holds phi^n):
        m * (phi^n - phi^(n-1)) / s_r on the network's grid, before the
        division by out_scale."""
        d = self._core_phi(solver.phi) - self._core_phi(phi_prev)
        return (self._coarsen(d) * self._net_mask(solver) * (1.0 / s_r)).to(torch.bfloat16).contiguous()

    @torch.no_grad()
    def predict(self, x2):
        x = torch.zeros(x2.shape[:3] + (16,), dtype=torch.bfloat16, device=x2.device)
        x[..., :2] = x2
        return self.net(x)

    @staticmethod
    def _periodic_images(phi, bounds):
        """The guard and image planes of periodic axes from the nodes they
        copy (applyboundaryconditions3d's order: x, then y, then z)."""
        for axis, lo in ((0, 0), (1, 2), (2, 4)):
            if bounds[lo] == 2 and bounds[lo + 1] == 2:
                n = phi.shape[axis] - 3
                sel = lambda i: (slice(None),) * axis + (i,)
                phi[sel(n + 1)] = phi[sel(1)]
                phi[sel(0)] = phi[sel(n)]
                phi[sel(n + 2)] = phi[sel(2)]

    # The guard keeps a guess only when its relative residual is at least
    # this many times below that of phi^(n-1). Measured: on the 128x128x256
    # training grid the guesses start 3.6-5.3x lower and save one V-cycle in
    # five; on 256x256x512 (network on the grid coarsened by two) they start
    # about 1.2x lower and cost 2-3 V-cycles.
    MIN_GAIN = 3.0

    @torch.no_grad()
    def guess(self, solver, guard=True):
        """Adds the predicted change, times the mask, to solver.phi (which
        holds phi^(n-1)) on the nodes 0..n-1, then copies the periodic
        images; the solver's boundary handling sets the rest.

        With guard, the relative residual of phi^(n-1) and of the guess are
        both measured, and phi^(n-1) is put back unless the guess starts at
        least MIN_GAIN times lower (so a state unlike the training snapshots,
        such as the first step after the initial solve, keeps phi^(n-1)).
        Returns (relres of phi^(n-1), relres of the guess, whether the guess
        was kept); without guard the residuals are not measured (None) and
        the guess is always kept. A call skipped by the back-off returns
        (None, None, False)."""
        self.calls += 1
        if guard and self._skip > 0:
            self._skip -= 1
            return None, None, False
        self.tried += 1
        r_plain = solver.relresidual() if guard else None
        x, s_r = self.inputs(solver)
        d = self.lowpass(self.predict(x))
        if self.factor > 1:
            d = torch.nn.functional.interpolate(d[None, None], scale_factor=self.factor, mode="trilinear",
                                                align_corners=False)[0, 0]
        d = d * self.node_mask(solver, self.out_margin)
        prev = solver.phi.clone() if guard else None
        interior = solver.phi[1:-2, 1:-2, 1:-2]
        interior.add_((d * (s_r * self.out_scale)).permute(2, 1, 0).to(torch.float64))
        self._periodic_images(solver.phi, solver.bounds)
        check_errors(solver.device)
        if not guard:
            return None, None, True
        r_learned = solver.relresidual()
        if r_learned * self.MIN_GAIN <= r_plain:
            return r_plain, r_learned, True
        solver.phi.copy_(prev)  # phi^(n-1) exactly
        self._skip = self.backoff - 1
        return r_plain, r_learned, False

    def state(self):
        return {"weights": {k: v.detach().to(torch.bfloat16).cpu() for k, v in self.net.state_dict().items()},
                "out_scale": self.out_scale, "smooth": self.smooth, "margin": self.margin,
                "out_margin": self.out_margin, "train_factor": getattr(self, "train_factor", self.factor)}

    @classmethod
    def load(cls, state, device="cuda", factor=None):
        """From state() or from a file written with torch.save(state()).
        factor defaults to the one the network was trained at."""
        if isinstance(state, str):
            state = torch.load(state, map_location="cpu")
        net = UNet3D(device=device)
        net.load_state_dict({k: v.float().to(device) for k, v in state["weights"].items()})
        tf = int(state.get("train_factor", 1))
        ws = cls(net, out_scale=state["out_scale"], smooth=state.get("smooth", "none"),
                 factor=tf if factor is None else factor, margin=state.get("margin", 2),
                 out_margin=state.get("out_margin", 6))
        ws.train_factor = tf
        return ws


def _bench_main():
    """python -m warp_b200.unet [--cin C --cout C --dhw D H W --reps N]:
    times wg_conv3_fwd (forward, bias, ReLU) on random bf16 data with CUDA
    events and prints the dense TFLOP/s (2*27*cin*cout per voxel)."""
    import argparse
    import json
    ap = argparse.ArgumentParser()
    ap.add_argument("--cin", type=int, default=64)
    ap.add_argument("--cout", type=int, default=64)
    ap.add_argument("--dhw", type=int, nargs=3, default=[128, 128, 128])
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args()
    D, H, W = a.dhw
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((D, H, W, a.cin), generator=g, device="cuda").to(torch.bfloat16)
    w = (torch.randn((27, a.cout, a.cin), generator=g, device="cuda") * 0.05).to(torch.bfloat16)
    b = torch.zeros(a.cout, device="cuda")
    y = conv3_fwd(x, w, b, relu=True)  # warm-up
    torch.cuda.synchronize()
    ms = []
    for _ in range(a.reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        conv3_fwd(x, w, b, relu=True, out=y)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    check_errors(x.device)
    flop = 2.0 * 27 * a.cin * a.cout * D * H * W
    best = min(ms)
    print(json.dumps({"kernel": "k_conv3_tile", "cin": a.cin, "cout": a.cout, "dhw": [D, H, W],
                      "ms": ms, "tflops_best": flop / (best * 1e-3) / 1e12,
                      "tflops_median": flop / (sorted(ms)[len(ms) // 2] * 1e-3) / 1e12}))


if __name__ == "__main__":
    _bench_main()
