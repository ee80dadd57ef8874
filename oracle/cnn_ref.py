"""CPU oracle (float64 NumPy) for the warm-start network's 3x3 convolution
products -- TEST INFRASTRUCTURE ONLY.  Layouts follow the kernels: x [N,H,W,C],
w [K,3,3,C], y [N,P,Q,K]; pad 1; output index p reads input rows
p*stride + r - 1 for taps r = 0..2."""
import numpy as np


def conv_out(n, stride):
    return n if stride == 1 else (n + 1) // 2


def _patches(xp, r, s, stride, P, Q):
    return xp[:, r:r + stride * (P - 1) + 1:stride, s:s + stride * (Q - 1) + 1:stride, :]


def forward(x, w, b, stride, relu):
    N, H, W, C = x.shape
    K = w.shape[0]
    P, Q = conv_out(H, stride), conv_out(W, stride)
    xp = np.pad(x.astype(np.float64), ((0, 0), (1, 1), (1, 1), (0, 0)))
    y = np.zeros((N, P, Q, K))
    for r in range(3):
        for s in range(3):
            y += np.einsum("npqc,kc->npqk", _patches(xp, r, s, stride, P, Q), w[:, r, s, :].astype(np.float64))
    y += b.astype(np.float64)
    return np.maximum(y, 0.0) if relu else y


def backward(x, w, g, stride, y_act=None):
    """Gradients of sum(g * y) with y = conv(x, w) + b (g masked by y_act > 0
    when given): returns (gx, gw, gb)."""
    N, H, W, C = x.shape
    K = w.shape[0]
    P, Q = conv_out(H, stride), conv_out(W, stride)
    g = g.astype(np.float64)
    if y_act is not None:
        g = g * (y_act > 0)
    xp = np.pad(x.astype(np.float64), ((0, 0), (1, 1), (1, 1), (0, 0)))
    gxp = np.zeros_like(xp)
    gw = np.zeros(w.shape)
    for r in range(3):
        for s in range(3):
            gw[:, r, s, :] = np.einsum("npqk,npqc->kc", g, _patches(xp, r, s, stride, P, Q))
            gxp[:, r:r + stride * (P - 1) + 1:stride, s:s + stride * (Q - 1) + 1:stride, :] += \
                np.einsum("npqk,kc->npqc", g, w[:, r, s, :].astype(np.float64))
    return gxp[:, 1:-1, 1:-1, :], gw, g.sum(axis=(0, 1, 2))
