"""ORACLE — test infrastructure only, never part of the product path.

FP64 numpy restatement of the warm-start CNN's operations (3x3 convolution,
zero padding, stride 1, NCHW; ReLU; residual output), the checker for the
CUDA kernels of sgd_b200/csrc/cnn.cu.  The reference has no counterpart (its
layers/layer.hh scaffold holds no convolution), so this follows the textbook
definitions.
"""
import numpy as np


def conv3x3(x, w, b=None):
    """x (N, Ci, H, W), w (Co, Ci, 3, 3) -> (N, Co, H, W)."""
    N, Ci, H, W = x.shape
    xp = np.zeros((N, Ci, H + 2, W + 2))
    xp[:, :, 1:-1, 1:-1] = x
    out = np.zeros((N, w.shape[0], H, W))
    for ky in range(3):
        for kx in range(3):
            out += np.einsum("nchw,oc->nohw", xp[:, :, ky:ky + H, kx:kx + W], w[:, :, ky, kx])
    if b is not None:
        out += b[None, :, None, None]
    return out


def conv3x3_grads(x, w, gout):
    """(d input, d weights, d bias) of sum(gout * conv3x3(x, w, b))."""
    N, Ci, H, W = x.shape
    xp = np.zeros((N, Ci, H + 2, W + 2))
    xp[:, :, 1:-1, 1:-1] = x
    gw = np.zeros(w.shape, dtype=np.float64)
    gxp = np.zeros_like(xp)
    for ky in range(3):
        for kx in range(3):
            gw[:, :, ky, kx] = np.einsum("nohw,nchw->oc", gout, xp[:, :, ky:ky + H, kx:kx + W])
            gxp[:, :, ky:ky + H, kx:kx + W] += np.einsum("nohw,oc->nchw", gout, w[:, :, ky, kx])
    return gxp[:, :, 1:-1, 1:-1], gw, gout.sum(axis=(0, 2, 3))


def network(x, ws, bs):
    """Residual net: ReLU after every layer but the last, output x + last."""
    acts = [x]
    h = x
    for k, (w, b) in enumerate(zip(ws, bs)):
        h = conv3x3(h, w, b)
        if k < len(ws) - 1:
            h = np.maximum(h, 0.0)
        acts.append(h)
    return x + h, acts


def network_grads(x, ws, bs, gy):
    """Parameter gradients of sum(gy * network(x))."""
    _, acts = network(x, ws, bs)
    g = gy.copy()
    gws, gbs = [None] * len(ws), [None] * len(ws)
    for k in reversed(range(len(ws))):
        if k < len(ws) - 1:
            g = g * (acts[k + 1] > 0)
        gx, gws[k], gbs[k] = conv3x3_grads(acts[k], ws[k], g)
        g = gx
    return gws, gbs
