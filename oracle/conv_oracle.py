"""FP64 CPU oracle of the 3x3x3 convolutions of the learned warm start.

TEST INFRASTRUCTURE ONLY: used by tests/ to check the tensor-core kernels
(forward, data gradient, weight gradient) and the network's gradients. The
learned warm start has no counterpart in the reference, so this oracle
restates the plain mathematics of a zero-padded 3x3x3 convolution.

Layouts follow the kernels: activations [D][H][W][C] (channels last),
weights [27][Cout][Cin] with tap t = 9*(dz+1) + 3*(dy+1) + (dx+1).
"""
import numpy as np

TAPS = [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def _shift(xp, dz, dy, dx, D, H, W):
    """x[z+dz, y+dy, x+dx] for all (z, y, x) from the 1-padded array xp."""
    return xp[1 + dz:1 + dz + D, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W]


def conv3_fwd(x, w, bias=None, relu=False):
    """y[v][co] = sum_t sum_ci x[v + off_t][ci] w[t][co][ci] (+bias, ReLU)."""
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    D, H, W, cin = x.shape
    cout = w.shape[1]
    xp = np.zeros((D + 2, H + 2, W + 2, cin))
    xp[1:-1, 1:-1, 1:-1] = x
    y = np.zeros((D, H, W, cout))
    for t, (dz, dy, dx) in enumerate(TAPS):
        y += _shift(xp, dz, dy, dx, D, H, W) @ w[t].T
    if bias is not None:
        y += np.asarray(bias, np.float64)
    if relu:
        y = np.maximum(y, 0.)
    return y


def conv3_dgrad(dy, w):
    """dx[u][ci] = sum_t sum_co dy[u - off_t][co] w[t][co][ci]."""
    dy = np.asarray(dy, np.float64)
    w = np.asarray(w, np.float64)
    D, H, W, cout = dy.shape
    cin = w.shape[2]
    dp = np.zeros((D + 2, H + 2, W + 2, cout))
    dp[1:-1, 1:-1, 1:-1] = dy
    dx_ = np.zeros((D, H, W, cin))
    for t, (dz, ddy, ddx) in enumerate(TAPS):
        dx_ += _shift(dp, -dz, -ddy, -ddx, D, H, W) @ w[t]
    return dx_


def conv3_wgrad(x, dy):
    """dw[t][co][ci] = sum_v dy[v][co] x[v + off_t][ci]."""
    x = np.asarray(x, np.float64)
    dy = np.asarray(dy, np.float64)
    D, H, W, cin = x.shape
    cout = dy.shape[3]
    xp = np.zeros((D + 2, H + 2, W + 2, cin))
    xp[1:-1, 1:-1, 1:-1] = x
    dw = np.zeros((27, cout, cin))
    d2 = dy.reshape(-1, cout)
    for t, (dz, ddy, ddx) in enumerate(TAPS):
        dw[t] = d2.T @ _shift(xp, dz, ddy, ddx, D, H, W).reshape(-1, cin)
    return dw


def flip_transpose(w):
    """Weights of the data-gradient convolution: w'[t][ci][co] = w[26-t][co][ci]."""
    w = np.asarray(w)
    return np.ascontiguousarray(w[::-1].transpose(0, 2, 1))
