"""Naive FP64 restatement of the surrogate's 3D convolution and its
gradients (the learned warm start has no counterpart in the reference).

TEST INFRASTRUCTURE ONLY: the checker for coffee_b200's BF16 tensor-core
convolution kernels.  Nothing in the library imports this module.

Layout: activations (N, D, H, W, C) channels last; weights (K, 27, C) with
tap t = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1); zero padding of one point,
stride 1 ("same" 3x3x3 convolution):

  y[n, z, y, x, k] = b[k] + sum_{t, c} x[n, z + dz, y + dy, x + dx, c] * w[k, t, c]
"""
from __future__ import annotations

import numpy as np

TAPS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def _shifted(x, dz, dy, dx):
    """x[n, z + dz, y + dy, x + dx, :] with zeros outside (N, D, H, W, C)."""
    out = np.zeros_like(x)
    D, H, W = x.shape[1:4]
    zs = slice(max(0, -dz), min(D, D - dz))
    ys = slice(max(0, -dy), min(H, H - dy))
    xs = slice(max(0, -dx), min(W, W - dx))
    zsrc = slice(max(0, dz), min(D, D + dz))
    ysrc = slice(max(0, dy), min(H, H + dy))
    xsrc = slice(max(0, dx), min(W, W + dx))
    out[:, zs, ys, xs, :] = x[:, zsrc, ysrc, xsrc, :]
    return out


def conv3d(x, w, b=None):
    x = np.asarray(x, np.float64)
    w = np.asarray(w, np.float64)
    y = np.zeros(x.shape[:4] + (w.shape[0],))
    for t, (dz, dy, dx) in enumerate(TAPS):
        y += _shifted(x, dz, dy, dx) @ w[:, t, :].T
    if b is not None:
        y += np.asarray(b, np.float64)
    return y


def conv3d_grad_input(dy, w):
    """dL/dx for dL/dy: the transposed convolution."""
    dy = np.asarray(dy, np.float64)
    w = np.asarray(w, np.float64)
    dx = np.zeros(dy.shape[:4] + (w.shape[2],))
    for t, (dz, dyy, dxx) in enumerate(TAPS):
        dx += _shifted(dy, -dz, -dyy, -dxx) @ w[:, t, :]
    return dx


def conv3d_grad_weight(dy, x):
    """dL/dw[k, t, c] = sum over points of dy[., k] x[. + offset(t), c]."""
    dy = np.asarray(dy, np.float64)
    x = np.asarray(x, np.float64)
    K, C = dy.shape[-1], x.shape[-1]
    dw = np.zeros((K, 27, C))
    flat_dy = dy.reshape(-1, K)
    for t, (dz, dyy, dxx) in enumerate(TAPS):
        dw[:, t, :] = flat_dy.T @ _shifted(x, dz, dyy, dxx).reshape(-1, C)
    return dw


def leaky(z, slope=0.1):
    return np.where(z > 0, z, slope * z)


def leaky_grad(z, slope=0.1):
    return np.where(z > 0, 1.0, slope)


def avgpool2(x):
    N, D, H, W, C = x.shape
    return x.reshape(N, D // 2, 2, H // 2, 2, W // 2, 2, C).mean(axis=(2, 4, 6))


def upsample2(x):
    return x.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)


def bf16(a):
    """Round to bfloat16 (nearest even) and back to float64."""
    a32 = np.asarray(a, np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unet_forward_backward(ws, bs, x, target, mask, slope=0.1):
    """FP64 restatement of coffee_b200.surrogate.UNet: forward pass, masked
    MSE loss and the gradients of every layer, rounding to bfloat16 exactly
    where the kernels store BF16 (weights, layer inputs, the activations and
    the dz that feed the convolutions).  ws[i] (K, 27, C), bs[i] (K,), x (N, D,
    H, W, 16) already BF16-valued.  Returns (loss, dws, dbs, output)."""
    w = [bf16(a) for a in ws]
    z1 = conv3d(x, w[0], bs[0]); a1 = bf16(leaky(z1, slope))
    z2 = conv3d(a1, w[1], bs[1]); a2 = bf16(leaky(z2, slope))
    p2 = bf16(avgpool2(a2))
    z3 = conv3d(p2, w[2], bs[2]); a3 = bf16(leaky(z3, slope))
    z4 = conv3d(a3, w[3], bs[3]); a4 = bf16(leaky(z4, slope))
    cat = np.concatenate([upsample2(a4), a2], axis=-1)
    z5 = conv3d(cat, w[4], bs[4]); a5 = bf16(leaky(z5, slope))
    out = conv3d(a5, w[5], bs[5])
    m = mask[..., None]
    count = float(mask.sum()) * out.shape[-1]
    diff = out - target
    loss = float((m * diff * diff).sum() / count)
    dout = 2.0 * m * diff / count
    dws, dbs = [None] * 6, [None] * 6

    def layer(i, dz, xin):
        dzb = bf16(dz)
        dbs[i] = dz.reshape(-1, dz.shape[-1]).sum(axis=0)
        dws[i] = conv3d_grad_weight(dzb, xin)
        return conv3d_grad_input(dzb, w[i])

    da5 = layer(5, dout, a5)
    dcat = layer(4, da5 * leaky_grad(z5, slope), cat)
    c2 = a4.shape[-1]
    du = dcat[..., :c2]
    da4 = du.reshape(du.shape[0], du.shape[1] // 2, 2, du.shape[2] // 2, 2, du.shape[3] // 2, 2,
                     c2).sum(axis=(2, 4, 6))
    da2 = dcat[..., c2:].copy()
    da3 = layer(3, da4 * leaky_grad(z4, slope), a3)
    dp2 = layer(2, da3 * leaky_grad(z3, slope), p2)
    da2 += upsample2(dp2) / 8.0
    da1 = layer(1, da2 * leaky_grad(z2, slope), a1)
    layer(0, da1 * leaky_grad(z1, slope), x)
    return loss, dws, dbs, out
