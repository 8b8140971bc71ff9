"""Tensor-core (tcgen05) BF16 convolutions against the FP64 oracle: forward
with bias/ReLU/mask/channel offset, data gradient through the mirrored
weights, weight gradient, and the U-Net's autograd gradients. Inputs are
bf16-representable, so the oracle sees exactly the kernel's operands; the
tolerance covers FP32 accumulation order and the bf16 rounding of outputs."""
import numpy as np
import pytest
import torch

from oracle import conv_oracle as co

pytestmark = pytest.mark.gpu


def _bf(a):
    return torch.as_tensor(a, dtype=torch.float32).to(torch.bfloat16)


def _rand(shape, seed, scale=1.0):
    g = torch.Generator().manual_seed(seed)
    return (torch.randn(shape, generator=g) * scale).to(torch.bfloat16)


@pytest.mark.parametrize("dims,cin,cout", [((5, 6, 40), 16, 16), ((4, 4, 33), 32, 64), ((3, 5, 7), 48, 128),
                                           ((8, 8, 16), 128, 32), ((3, 4, 18), 64, 192)])
def test_conv3_fwd_matches_oracle(dims, cin, cout):
    from warp_b200 import unet
    D, H, W = dims
    x = _rand((D, H, W, cin), 1)
    w = _rand((27, cout, cin), 2, 0.2)
    b = torch.randn(cout, generator=torch.Generator().manual_seed(3))
    y = unet.conv3_fwd(x.cuda(), w.cuda(), b.cuda(), relu=True)
    unet.check_errors(y.device)
    ref = co.conv3_fwd(x.float().numpy(), w.float().numpy(), b.numpy(), relu=True)
    got = y.float().cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-2 * np.max(np.abs(ref)) + 1e-2


def test_conv3_fwd_offset_and_mask():
    from warp_b200 import unet
    D, H, W, cin, cout = 4, 5, 30, 16, 32
    x = _rand((D, H, W, cin), 4)
    w = _rand((27, cout, cin), 5, 0.2)
    m = _rand((D, H, W, cout), 6)
    out = torch.full((D, H, W, 48), 7.0, dtype=torch.bfloat16, device="cuda")
    unet.conv3_fwd(x.cuda(), w.cuda(), None, relu=False, out=out, yoff=16, mask=m.cuda())
    unet.check_errors(out.device)
    ref = co.conv3_fwd(x.float().numpy(), w.float().numpy()) * (m.float().numpy() > 0)
    got = out.float().cpu().numpy()
    assert np.all(got[..., :16] == 7.0)
    assert np.max(np.abs(got[..., 16:] - ref)) <= 1e-2 * np.max(np.abs(ref)) + 1e-2


@pytest.mark.parametrize("dims,cin,cout", [((5, 6, 40), 16, 16), ((3, 5, 7), 48, 128)])
def test_conv3_fwd_f32_output(dims, cin, cout):
    """The FP32-output form: within FP32 accumulation error of the FP64
    oracle (no bf16 rounding), and rounded to bf16 it equals the bf16-output
    form bit for bit."""
    from warp_b200 import unet
    D, H, W = dims
    x = _rand((D, H, W, cin), 11)
    w = _rand((27, cout, cin), 12, 0.2)
    b = torch.randn(cout, generator=torch.Generator().manual_seed(13))
    yf = unet.conv3_fwd(x.cuda(), w.cuda(), b.cuda(), relu=True, out_dtype=torch.float32)
    yb = unet.conv3_fwd(x.cuda(), w.cuda(), b.cuda(), relu=True)
    unet.check_errors(yf.device)
    assert yf.dtype == torch.float32
    ref = co.conv3_fwd(x.float().numpy(), w.float().numpy(), b.numpy(), relu=True)
    got = yf.cpu().numpy()
    assert np.max(np.abs(got - ref)) <= 1e-5 * np.max(np.abs(ref)) + 1e-5
    assert torch.equal(yf.to(torch.bfloat16), yb)


@pytest.mark.parametrize("cin,cout", [(32, 16), (192, 64), (16, 16), (48, 16), (64, 128), (128, 128), (96, 32)])
def test_conv3_dgrad_and_wgrad_match_oracle(cin, cout):
    from warp_b200 import unet
    D, H, W = 6, 5, 20
    x = _rand((D, H, W, cin), 7)
    w = _rand((27, cout, cin), 8, 0.2)
    dy = _rand((D, H, W, cout), 9)
    dx = unet.conv3_fwd(dy.cuda(), unet.flip_transpose(w.cuda()), None, relu=False)
    dw = unet.conv3_wgrad(x.cuda(), dy.cuda())
    unet.check_errors(dx.device)
    # fixed-order partial sums: the same bits on a second run
    assert torch.equal(unet.conv3_wgrad(x.cuda(), dy.cuda()), dw)
    rdx = co.conv3_dgrad(dy.float().numpy(), w.float().numpy())
    rdw = co.conv3_wgrad(x.float().numpy(), dy.float().numpy())
    assert np.max(np.abs(dx.float().cpu().numpy() - rdx)) <= 1e-2 * np.max(np.abs(rdx)) + 1e-2
    # fp32 accumulation of exact bf16 products: only summation order differs
    assert np.max(np.abs(dw.cpu().numpy() - rdw)) <= 1e-4 * np.max(np.abs(rdw))


def test_unet_gradients_against_oracle_chain():
    """One conv + ReLU + sum loss through autograd equals the oracle's
    chain rule (weights, bias, input)."""
    from warp_b200 import unet
    D, H, W, cin, cout = 4, 4, 16, 16, 32
    x = _rand((D, H, W, cin), 10).cuda().requires_grad_(True)
    w = (torch.randn(27, cout, cin, generator=torch.Generator().manual_seed(11)) * 0.2)
    w = w.to(torch.bfloat16).float().cuda().requires_grad_(True)
    b = torch.zeros(cout, device="cuda", requires_grad=True)
    y = unet.conv3(x, w, b, relu=True)
    g = _rand((D, H, W, cout), 12).cuda()
    (y.float() * g.float()).sum().backward()
    unet.check_errors(y.device)
    xn, wn = x.detach().float().cpu().numpy(), w.detach().cpu().numpy()
    pre = co.conv3_fwd(xn, wn)
    # the ReLU mask comes from the kernel's bf16 output; it must agree with
    # the oracle's pre-activation sign wherever that is not within rounding
    # of zero, and the chain rule is checked for that mask
    act = y.detach().float().cpu().numpy() > 0
    near0 = np.abs(pre) <= 1e-2 * np.max(np.abs(pre))
    assert np.all((act == (pre > 0)) | near0)
    gz = g.float().cpu().numpy() * act
    rdw = co.conv3_wgrad(xn, gz)
    rdb = gz.sum(axis=(0, 1, 2))
    rdx = co.conv3_dgrad(gz, wn)
    assert np.max(np.abs(b.grad.cpu().numpy() - rdb)) <= 1e-3 * np.max(np.abs(rdb))
    assert np.max(np.abs(w.grad.cpu().numpy() - rdw)) <= 2e-2 * np.max(np.abs(rdw))
    assert np.max(np.abs(x.grad.float().cpu().numpy() - rdx)) <= 2e-2 * np.max(np.abs(rdx))
