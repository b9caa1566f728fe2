"""FP64 numpy restatement of the warm-start network's 3x3x3 convolution and
its gradients (TEST INFRASTRUCTURE ONLY).

The reference has no counterpart (its only network is an unrelated MLP
surrogate); this oracle checks the tensor-core kernels' forward, input
gradient and weight gradient directly from the definition:
    y[v, co] = b[co] + sum_{tap, ci} x[v + tap - 1, ci] w[co, tap, ci]
with zero padding, tap = 9 kd + 3 kh + kw, tensors NDHWC.
"""
import numpy as np


def im2col(x):
    """(N,D,H,W,C) -> (N*D*H*W, 27*C), column index tap*C + ci."""
    N, D, H, W, C = x.shape
    xp = np.zeros((N, D + 2, H + 2, W + 2, C), dtype=np.float64)
    xp[:, 1:-1, 1:-1, 1:-1] = x
    cols = []
    for kd in range(3):
        for kh in range(3):
            for kw in range(3):
                cols.append(xp[:, kd:kd + D, kh:kh + H, kw:kw + W, :].reshape(-1, C))
    return np.concatenate(cols, axis=1)


def conv3d(x, w, b=None, relu=False):
    """x (N,D,H,W,Cin), w (Cout,27,Cin) -> (N,D,H,W,Cout)."""
    N, D, H, W, _ = x.shape
    Cout = w.shape[0]
    y = im2col(x) @ w.reshape(Cout, -1).T.astype(np.float64)
    if b is not None:
        y = y + b[None, :]
    if relu:
        y = np.maximum(y, 0.0)
    return y.reshape(N, D, H, W, Cout)


def conv3d_backward(x, w, dy, y=None, relu=False):
    """Gradients (dx, dw, db) of sum(dy * conv3d(x, w, b, relu))."""
    N, D, H, W, Cin = x.shape
    Cout = w.shape[0]
    dz = dy.astype(np.float64)
    if relu:
        dz = np.where(y > 0, dz, 0.0)
    dz2 = dz.reshape(-1, Cout)
    dw = (dz2.T @ im2col(x)).reshape(Cout, 27, Cin)
    db = dz2.sum(axis=0)
    # dx[v, ci] = sum_{tap, co} dz[v - (tap - 1), co] w[co, tap, ci]: a conv of dz
    # with the tap-flipped, transposed kernel
    wt = np.flip(w, axis=1).transpose(2, 1, 0)  # (Cin, 27, Cout)
    dx = conv3d(dz, wt)
    return dx, dw, db
