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


def conv3_fwd(x, w, bias=None, relu=False, out=None, yoff=0, mask=None):
    """x: [D,H,W,Cin] bf16; w: [27,Cout,Cin] bf16; bias fp32 [Cout] or None.
    Writes channels yoff..yoff+Cout-1 of `out` ([D,H,W,Ctot] bf16)."""
    D, H, W, cin = x.shape
    cout = w.shape[1]
    assert x.dtype == torch.bfloat16 and w.dtype == torch.bfloat16 and x.is_contiguous() and w.is_contiguous()
    assert w.shape == (27, cout, cin)
    if out is None:
        out = torch.empty((D, H, W, cout), dtype=torch.bfloat16, device=x.device)
    assert out.is_contiguous() and out.shape[:3] == (D, H, W)
    if mask is not None:
        assert mask.is_contiguous() and mask.shape[:3] == (D, H, W)
    err = _errbuf(x.device)
    _lib.check(_lib.lib.wg_conv3_fwd(
        x.data_ptr(), D, H, W, cin, w.data_ptr(), bias.data_ptr() if bias is not None else None, cout,
        out.data_ptr(), out.shape[3], yoff, mask.data_ptr() if mask is not None else None,
        mask.shape[3] if mask is not None else 0, int(relu), err.data_ptr(), _stream(x.device)))
    return out


def conv3_wgrad(x, dy):
    """dW[t][co][ci] = sum_v dy[v][co] x[v+off_t][ci] (fp32)."""
    D, H, W, cin = x.shape
    cout = dy.shape[3]
    xT = x.permute(3, 0, 1, 2).contiguous()
    dyT = dy.permute(3, 0, 1, 2).contiguous()
    dw = torch.zeros((27, cout, cin), dtype=torch.float32, device=x.device)
    err = _errbuf(x.device)
    _lib.check(_lib.lib.wg_conv3_wgrad(xT.data_ptr(), dyT.data_ptr(), D, H, W, cin, cout, dw.data_ptr(),
                                       err.data_ptr(), _stream(x.device)))
    return dw


def flip_transpose(w):
    """Weights of the data-gradient convolution: w'[t][ci][co] = w[26-t][co][ci]."""
    return w.flip(0).transpose(1, 2).contiguous()


class _Conv3(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, w, b, relu):
        wb = w.to(torch.bfloat16).contiguous()
        y = conv3_fwd(x.contiguous(), wb, b.float().contiguous(), relu=relu)
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
        return dx, dw, db, None


def conv3(x, w, b, relu=True):
    return _Conv3.apply(x, w, b, relu)


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

    def c(self, name, x, relu=True):
        return conv3(x, self.w[name], self.b[name], relu)

    def forward(self, x):
        """x: [D,H,W,16] bf16 (2 used channels); returns [D,H,W] fp32."""
        e1 = self.c("e1b", self.c("e1a", x))
        e2 = self.c("e2b", self.c("e2a", _pool(e1)))
        e3 = self.c("e3b", self.c("e3a", _pool(e2)))
        m = self.c("m2", self.c("m1", _pool(e3)))
        d3 = self.c("d3b", self.c("d3a", torch.cat([_up(m), e3], dim=3)))
        d2 = self.c("d2b", self.c("d2a", torch.cat([_up(d3), e2], dim=3)))
        d1 = self.c("d1b", self.c("d1a", torch.cat([_up(d2), e1], dim=3)))
        return self.c("out", d1, relu=False)[..., 0].float()


class WarmStart:
    """Scaling around the solver's arrays. The network sees, on the nodes
    0..nx-1, 0..ny-1, 0..nz-1 (z, y, x order), phi^(n-1)/s and
    rho * rho_factor / s with s = max|phi^(n-1)|, and predicts
    out_scale * (phi^n - phi^(n-1)) / s. With rho_factor ~ dx^2/eps0 both
    inputs are O(1) whatever the beam current."""

    def __init__(self, net, rho_factor, out_scale=30.0):
        self.net = net
        self.rho_factor = float(rho_factor)
        self.out_scale = float(out_scale)

    def _core(self, rho, phi):
        return rho[:-1, :-1, :-1].permute(2, 1, 0), phi[1:-2, 1:-2, 1:-2].permute(2, 1, 0)

    def inputs(self, rho, phi_prev):
        """rho: solver.rho [nx+1,ny+1,nz+1] (Fortran view); phi_prev: solver.phi
        [nx+3,ny+3,nz+3]. Returns ([D,H,W,2] bf16, s)."""
        r, p = self._core(rho, phi_prev)
        s = float(p.abs().max().item()) or 1.0
        x = torch.empty(r.shape + (2,), dtype=torch.bfloat16, device=rho.device)
        x[..., 0] = (r * (self.rho_factor / s)).to(torch.bfloat16)
        x[..., 1] = (p / s).to(torch.bfloat16)
        return x, s

    def pair(self, rho, phi_prev, phi):
        """Training pair (inputs, target) of one solved step."""
        x, s = self.inputs(rho, phi_prev)
        _, p0 = self._core(rho, phi_prev)
        _, p1 = self._core(rho, phi)
        y = ((p1 - p0) * (self.out_scale / s)).to(torch.bfloat16).contiguous()
        return x.contiguous(), y

    @torch.no_grad()
    def predict(self, x2):
        x = torch.zeros(x2.shape[:3] + (16,), dtype=torch.bfloat16, device=x2.device)
        x[..., :2] = x2
        return self.net(x)

    @torch.no_grad()
    def guess(self, solver):
        """Adds the predicted change to solver.phi (which holds phi^(n-1)) on
        the nodes 0..n-1; the solver's boundary handling sets the rest."""
        x, s = self.inputs(solver.rho, solver.phi)
        d = self.predict(x)
        interior = solver.phi[1:-2, 1:-2, 1:-2]
        interior.add_((d * (s / self.out_scale)).permute(2, 1, 0).to(torch.float64))
        check_errors(solver.device)
