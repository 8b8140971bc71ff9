"""Host logic of the learned guess that needs no GPU: the back-off after a
rejected guess skips the network without touching the solver, and the
state round trip keeps the masks, the factor it was trained at and the
filter."""
import torch

from warp_b200.unet import UNet3D, WarmStart


class _NoSolver:
    """Any use of the solver fails the test."""

    def __getattr__(self, name):
        raise AssertionError("the solver was used: %s" % name)


def test_backoff_skips_the_network_and_counts():
    ws = WarmStart(None, backoff=3)
    ws._skip = 2
    s = _NoSolver()
    assert ws.guess(s) == (None, None, False)
    assert ws.guess(s) == (None, None, False)
    assert ws._skip == 0
    assert (ws.calls, ws.tried) == (2, 0)


def test_state_round_trip():
    net = UNet3D(device="cpu")
    ws = WarmStart(net, out_scale=2.5, smooth="box2", factor=1, margin=3, out_margin=5)
    ws.train_factor = 2
    st = ws.state()
    back = WarmStart.load(st, device="cpu")
    assert (back.out_scale, back.smooth, back.margin, back.out_margin, back.factor, back.train_factor) == \
        (2.5, "box2", 3, 5, 2, 2)
    assert WarmStart.load(st, device="cpu", factor=4).factor == 4
    for k, v in net.state_dict().items():
        assert torch.equal(back.net.state_dict()[k], v.to(torch.bfloat16).float()), k
