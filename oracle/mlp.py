"""CPU restatement of the learned-padding pieces (test infrastructure only:
imported by tests/ to check the GPU kernels).

- labels(): the method's expected axis covariance C_P(h) as a direct FP64
  cosine sum of the axis spectrum, the padding error max_h |C_P - C_32N| and
  the bisection for the smallest P and overlap width W (the rules of
  scarl_b200/csrc/mlp.cu, restated with numpy).
- mlp_forward_backward(): the 16 -> 64 -> 64 -> 2 ReLU network with BF16
  rounding (round to nearest even) of weights, inputs and hidden activations,
  products summed in FP64 (the GPU sums in FP32), MSE loss and gradients.
"""
import math

import numpy as np

IN, HID, OUT = 16, 64, 2


def bf16(x):
    """Round float32 values to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    W1 = p[o:o + HID * IN].reshape(HID, IN); o += HID * IN
    b1 = p[o:o + HID]; o += HID
    W2 = p[o:o + HID * HID].reshape(HID, HID); o += HID * HID
    b2 = p[o:o + HID]; o += HID
    W3 = p[o:o + OUT * HID].reshape(OUT, HID); o += OUT * HID
    b3 = p[o:o + OUT]
    return W1, b1, W2, b2, W3, b3


def mlp_forward(p, X, rounding=True):
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(p)
    x = r(X)
    h1 = r(np.maximum(x @ r(W1).T + b1, 0.0))
    h2 = r(np.maximum(h1 @ r(W2).T + b2, 0.0))
    return x, h1, h2, h2 @ r(W3).T + b3


def mlp_forward_backward(p, X, T, rounding=True):
    """Loss and gradient; rounding=False drops the BF16 roundings (exact
    FP64 network, for checking the backward formulas by finite differences)."""
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(p)
    n = len(X)
    x, h1, h2, y = mlp_forward(p, X, rounding)
    e = y - np.asarray(T, dtype=np.float64)
    loss = float(np.sum(e * e) / n)
    dy = 2.0 * e / n
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    d2 = (dy @ r(W3)) * (h2 > 0)
    gW2 = d2.T @ h1
    gb2 = d2.sum(0)
    d1 = (d2 @ r(W2)) * (h1 > 0)
    gW1 = d1.T @ x
    gb1 = d1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


# ---------------------------------------------------------------------------
# labels
# ---------------------------------------------------------------------------
def axis_spectrum(corrMod, nu, ell, f):
    if corrMod == 1:
        return np.exp(-math.pi * ell * ell * f * f)
    v = 0.5 if corrMod == 3 else nu
    a = ell * math.gamma(v) / (2.0 * math.sqrt(math.pi) * math.gamma(v + 0.5))
    return (1.0 + 4.0 * math.pi ** 2 * a * a * f * f) ** (-(v + 0.5))


def method_cov(corrMod, nu, ell, N, P):
    """Expected axis covariance of the padded method, lags 0..N-1."""
    k = np.arange(0, P // 2 + 1)
    s = axis_spectrum(corrMod, nu, ell, k / P)
    w = np.full(len(k), 2.0)
    w[0] = 1.0
    if P % 2 == 0:
        w[-1] = 1.0
    h = np.arange(N)
    c = np.cos(2.0 * math.pi * np.outer(h, k) / P) @ (w * s)
    return c / np.sum(w * s)


def pad_error(corrMod, nu, ell, N, P):
    return float(np.max(np.abs(method_cov(corrMod, nu, ell, N, P) -
                               method_cov(corrMod, nu, ell, N, 32 * N))))


def labels(corrMod, nu, ell, N, tol=0.01):
    ref = method_cov(corrMod, nu, ell, N, 32 * N)
    err = lambda P: float(np.max(np.abs(method_cov(corrMod, nu, ell, N, P) - ref)))
    lo, hi = N, 16 * N
    sat = err(hi) > tol
    if err(lo) <= tol:
        hi = lo
    while hi - lo > 1:
        mid = (lo + hi) // 2
        if err(mid) <= tol:
            hi = mid
        else:
            lo = mid
    h = np.arange(N)

    def oerr(W):
        t = np.minimum(h / (W - 1), 1.0)
        return float(np.max((1.0 - np.cos(0.5 * math.pi * t)) * np.abs(ref)))

    wl, wh = 2, N
    if oerr(wl) <= tol:
        wh = wl
    while wh - wl > 1:
        mid = (wl + wh) // 2
        if oerr(mid) <= tol:
            wh = mid
        else:
            wl = mid
    return hi, wh, int(sat), err
