"""CPU restatement (numpy, FP32) of the learned coarse-correction network.

TEST INFRASTRUCTURE ONLY: the checker for the CUDA CNN kernels
(samrai_b200/csrc/fac_cnn.cu).  The network has no counterpart in the
reference; it is specified by the task: four 3x3x3 convolutions
1 -> 16 -> 16 -> 16 -> 1 channels, ReLU after the first three, no biases,
zero padding ("same"), BF16 weights and activations with FP32 accumulation.

Layouts match the GPU: activations [n, z, y, x, c] (channels last), weights
W1 [27, 16] (tap, out), W2/W3 [27, 16, 16] (tap, in, out), W4 [27, 16]
(tap, in); tap t = (dz+1)*9 + (dy+1)*3 + (dx+1).
"""
from __future__ import annotations

import numpy as np

OFFSETS = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]


def bf16(a: np.ndarray) -> np.ndarray:
    """Round FP32 to BF16 (round to nearest even), returned as FP32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounding = ((u >> 16) & 1) + 0x7FFF
    u = ((u + rounding) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def _shift(x, dz, dy, dx):
    """y[n, z, y, x] = x[n, z+dz, y+dy, x+dx] with zero padding."""
    out = np.zeros_like(x)
    n, S0, S1, S2 = x.shape[:4]
    zs = slice(max(0, -dz), S0 - max(0, dz))
    ys = slice(max(0, -dy), S1 - max(0, dy))
    xs = slice(max(0, -dx), S2 - max(0, dx))
    zd = slice(max(0, dz), S0 - max(0, -dz))
    yd = slice(max(0, dy), S1 - max(0, -dy))
    xd = slice(max(0, dx), S2 - max(0, -dx))
    out[:, zs, ys, xs] = x[:, zd, yd, xd]
    return out


def conv(x, w):
    """x [n,S,S,S,cin], w [27,cin,cout] -> [n,S,S,S,cout] (FP32 accumulate)."""
    out = np.zeros(x.shape[:4] + (w.shape[2],), dtype=np.float32)
    for t, (dz, dy, dx) in enumerate(OFFSETS):
        out += np.tensordot(_shift(x, dz, dy, dx), w[t], axes=([4], [0])).astype(np.float32)
    return out


def conv_bwd_data(dy, w):
    """Gradient w.r.t. the input of conv: dx[c] = sum_t dy[c - off_t] w[t]^T."""
    out = np.zeros(dy.shape[:4] + (w.shape[1],), dtype=np.float32)
    for t, (dz, dy_, dx) in enumerate(OFFSETS):
        out += np.tensordot(_shift(dy, -dz, -dy_, -dx), w[t], axes=([4], [1])).astype(np.float32)
    return out


def conv_bwd_weight(x, dy):
    """dw[t, cin, cout] = sum_cells x[cell + off_t, cin] dy[cell, cout]."""
    cin, cout = x.shape[4], dy.shape[4]
    dw = np.zeros((27, cin, cout), dtype=np.float32)
    d2 = dy.reshape(-1, cout).astype(np.float64)
    for t, (dz, dy_, dx) in enumerate(OFFSETS):
        xs = _shift(x, dz, dy_, dx).reshape(-1, cin).astype(np.float64)
        dw[t] = (xs.T @ d2).astype(np.float32)
    return dw


class CNN:
    """Weights as FP32 masters; every forward rounds weights and stored
    activations to BF16 like the GPU kernels."""

    def __init__(self, w1, w2, w3, w4, rounding=True):
        self.w = [np.asarray(w, dtype=np.float32) for w in (w1, w2, w3, w4)]
        self.r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float32))

    @staticmethod
    def init(seed=0, width=16, rounding=True):
        rng = np.random.default_rng(seed)
        def he(cin, cout):
            return (rng.standard_normal((27, cin, cout)) * np.sqrt(2.0 / (27 * cin))).astype(np.float32)
        return CNN(he(1, width)[:, 0, :], he(width, width), he(width, width), he(width, 1)[:, :, 0],
                   rounding=rounding)

    def forward(self, x0):
        """x0 [n,S,S,S] -> (prediction [n,S,S,S], stored activations)."""
        r = self.r
        w1, w2, w3, w4 = [r(w) for w in self.w]
        a0 = r(x0)[..., None]
        a1 = r(np.maximum(conv(a0, w1[:, None, :]), 0.0))
        a2 = r(np.maximum(conv(a1, w2), 0.0))
        a3 = r(np.maximum(conv(a2, w3), 0.0))
        y = conv(a3, w4[:, :, None])[..., 0]
        return y, (a0, a1, a2, a3)

    def loss_and_grads(self, x0, target, mask):
        """Masked mean squared error and its gradients (FP32 masters)."""
        r = self.r
        w1, w2, w3, w4 = [r(w) for w in self.w]
        y, (a0, a1, a2, a3) = self.forward(x0)
        m = float(mask.sum())
        diff = (y - target) * mask
        loss = float((diff.astype(np.float64) ** 2).sum() / m)
        dy4 = (2.0 / m * diff).astype(np.float32)[..., None]
        g4 = conv_bwd_weight(a3, dy4)[:, :, 0]
        d3 = r(conv_bwd_data(dy4, w4[:, :, None]) * (a3 > 0))
        g3 = conv_bwd_weight(a2, d3)
        d2 = r(conv_bwd_data(d3, w3) * (a2 > 0))
        g2 = conv_bwd_weight(a1, d2)
        d1 = r(conv_bwd_data(d2, w2) * (a1 > 0))
        g1 = conv_bwd_weight(a0, d1)[:, 0, :]
        return loss, [g1, g2, g3, g4]
