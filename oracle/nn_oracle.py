"""FP64 numpy restatement of the learned initialiser's network (forward,
mean-squared-error loss and backward pass) -- the checker of the library's
BF16 training kernels (gctffind_b200/csrc/gcf_nn.cu, gcf_learned.cpp).

TEST INFRASTRUCTURE ONLY: the gradient-check tests import it; the product
package never does.

The network, parameters in the library's flat order (weights [out][in]
row-major, then the bias; `in` in the library's im2col column order):
  conv1 4x4 stride 4 on the 256 x 256 x 1 polar spectrum -> 64 x 64 x 16
        (column kk = 4 * ky + kx)
  conv2, conv3, conv4 3x3 stride 2 pad 1, channel-last -> 32x32x32,
        16x16x32, 8x8x32 (column (3 * ky + kx) * C + c)
  fc1 [profile 256 | conv4 flattened (y, x, c)] 2304 -> 256, fc2 256 -> 128,
  fc3 128 -> 3; ReLU after every layer but fc3.
Loss: mean over the batch and the 3 outputs of (pred - target)^2.

The library multiplies BF16 copies of the weights; pass bf16_weights=True
(the default) to use the same rounded values here, so the comparison
isolates the rounding of the activations.  emulate_bf16=True also rounds to
BF16 wherever the library stores BF16 (gctffind_b200/csrc/gcf_learned.cpp
nn_forward / nn_backward): every ReLU output, the loss gradient dpred, and
each layer's masked input gradient (after the col2im sums for the
convolutions); products and sums stay FP64, so what remains is the
library's FP32 accumulation.
"""
from __future__ import annotations

import numpy as np

LAYERS = [(16, 16), (32, 144), (32, 288), (32, 288), (256, 2304), (128, 256), (3, 128)]


def param_count() -> int:
    return sum(o * i + o for o, i in LAYERS)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), as float64."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params, bf16_weights=True):
    out, off = [], 0
    p = np.asarray(params, np.float64)
    for o, i in LAYERS:
        w = p[off: off + o * i].reshape(o, i)
        b = p[off + o * i: off + o * i + o]
        out.append((bf16(w) if bf16_weights else w, b))
        off += o * i + o
    return out


def _im2col3(x):
    """x [B, H, W, C] -> cols [B, H/2, W/2, 9C] of a 3x3 stride-2 pad-1 conv."""
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C), x.dtype)
    xp[:, 1:H + 1, 1:W + 1, :] = x
    OH, OW = H // 2, W // 2
    parts = []
    for ky in range(3):
        for kx in range(3):
            parts.append(xp[:, ky: ky + 2 * OH: 2, kx: kx + 2 * OW: 2, :])
    return np.concatenate(parts, axis=-1)


def _col2im3(dcols, H, W, C):
    B, OH, OW, _ = dcols.shape
    dxp = np.zeros((B, H + 2, W + 2, C), dcols.dtype)
    for ky in range(3):
        for kx in range(3):
            k = 3 * ky + kx
            dxp[:, ky: ky + 2 * OH: 2, kx: kx + 2 * OW: 2, :] += dcols[..., k * C:(k + 1) * C]
    return dxp[:, 1:H + 1, 1:W + 1, :]


def forward_backward(params, x1, x2, target, bf16_weights=True, emulate_bf16=False):
    """Returns (loss, flat gradients, predictions)."""
    P = unpack(params, bf16_weights)
    q = bf16 if emulate_bf16 else (lambda v: v)
    x1 = np.asarray(x1, np.float64)
    x2 = np.asarray(x2, np.float64)
    t = np.asarray(target, np.float64)
    B = x1.shape[0]
    relu = lambda z: np.maximum(z, 0.0)
    # conv1: 4x4 stride-4 patches
    c1 = x2.reshape(B, 64, 4, 64, 4).transpose(0, 1, 3, 2, 4).reshape(B, 64, 64, 16)
    y1 = q(relu(c1 @ P[0][0].T + P[0][1]))
    c2 = _im2col3(y1)
    y2 = q(relu(c2 @ P[1][0].T + P[1][1]))
    c3 = _im2col3(y2)
    y3 = q(relu(c3 @ P[2][0].T + P[2][1]))
    c4 = _im2col3(y3)
    y4 = q(relu(c4 @ P[3][0].T + P[3][1]))
    h0 = np.concatenate([x1, y4.reshape(B, 2048)], axis=1)
    h1 = q(relu(h0 @ P[4][0].T + P[4][1]))
    h2 = q(relu(h1 @ P[5][0].T + P[5][1]))
    pred = h2 @ P[6][0].T + P[6][1]
    d = pred - t
    loss = float((d * d).mean())
    g = [None] * 7

    def lin_grad(k, dz, x):
        g[k] = (dz.reshape(-1, dz.shape[-1]).T @ x.reshape(-1, x.shape[-1]), dz.reshape(-1, dz.shape[-1]).sum(0))
        return dz @ P[k][0]

    dz = q(2.0 * d / (3.0 * B))
    dh2 = q(lin_grad(6, dz, h2) * (h2 > 0))
    dh1 = q(lin_grad(5, dh2, h1) * (h1 > 0))
    dh0 = lin_grad(4, dh1, h0)
    dy4 = q(dh0[:, 256:].reshape(B, 8, 8, 32) * (y4 > 0))
    dc4 = lin_grad(3, dy4, c4)
    dy3 = q(_col2im3(dc4, 16, 16, 32) * (y3 > 0))
    dc3 = lin_grad(2, dy3, c3)
    dy2 = q(_col2im3(dc3, 32, 32, 32) * (y2 > 0))
    dc2 = lin_grad(1, dy2, c2)
    dy1 = q(_col2im3(dc2, 64, 64, 16) * (y1 > 0))
    lin_grad(0, dy1, c1)
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in g])
    return loss, flat, pred


def split(flat):
    """Per-layer (weights, bias) views of a flat vector."""
    out, off = [], 0
    for o, i in LAYERS:
        out.append((flat[off: off + o * i].reshape(o, i), flat[off + o * i: off + o * i + o]))
        off += o * i + o
    return out


def polar_inputs(half, px):
    """The network inputs of one background-removed half spectrum
    `half` [tile][tile/2+1] (DC at (0, tile/2)) of pixel size px, as the
    library bins them (gctffind_b200/csrc/gcf_nn.cu k_nn_input): pixels with
    s^2 in [1/1600, 1/12.25) 1/A^2 go to s^2 bin k (256 uniform bins) and
    angle bin t = (atan2(fy, fx) + pi/2) * 256 / pi; x2[t][k] and x1[k] are
    the bins' means, standardised (population variance) over non-empty bins,
    empty bins 0.  Bin indices are computed in float32 like the library's;
    x2's means are rounded to BF16 before standardisation, as the library
    stores them.  Returns (x1 [256], x2 [256][256]) in float64."""
    half = np.asarray(half)
    cy, cx = half.shape
    tile = cy
    f32 = np.float32
    y, x = np.mgrid[0:cy, 0:cx]
    fx = x.astype(f32) / f32(tile)
    fy = (y - cy // 2).astype(f32) / f32(tile)
    inv_px2 = f32(1.0) / (f32(px) * f32(px))
    s2 = (fx * fx + fy * fy) * inv_px2
    s2lo, s2hi = f32(1.0) / f32(1600.0), f32(1.0) / f32(12.25)
    ds2 = (s2hi - s2lo) / f32(256.0)
    m = (s2 >= s2lo) & (s2 < s2hi)
    k = np.clip(((s2 - s2lo) / ds2).astype(np.int64), 0, 255)[m]
    ang = np.arctan2(fy.astype(np.float64), fx.astype(np.float64)) + 0.5 * np.pi
    t = np.clip((ang * (256.0 / np.pi)).astype(np.int64), 0, 255)[m]
    v = half.astype(np.float64)[m]

    def standardise(s, c, rounded):
        mean = np.where(c > 0, s / np.maximum(c, 1), 0.0)
        nz = c > 0
        mu = mean[nz].mean() if nz.any() else 0.0
        var = (mean[nz] ** 2).mean() - mu * mu if nz.any() else 0.0
        inv = 1.0 / np.sqrt(var) if var > 1e-30 else 0.0
        base = bf16(mean) if rounded else mean
        return np.where(nz, (base - mu) * inv, 0.0)

    c1 = np.bincount(k, minlength=256).astype(np.float64)
    s1 = np.bincount(k, weights=v, minlength=256)
    cell = t * 256 + k
    c2 = np.bincount(cell, minlength=65536).astype(np.float64)
    s2m = np.bincount(cell, weights=v, minlength=65536)
    return standardise(s1, c1, False), standardise(s2m, c2, True).reshape(256, 256)
