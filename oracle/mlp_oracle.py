"""ORACLE INFRASTRUCTURE (test-only): CPU restatement of the surrogate
network's forward and backward pass (unicorn_b200/csrc/mlp.cuh,
mlp_gemm.cuh), in float64 with the device's BF16 rounding points, for
checking the tensor-core gradients. Never used by the product.

Layers 64 -> 256 (GELU) -> 256 (GELU) -> 256 (GELU) -> 256 (GELU) -> 64
(linear), GELU in its tanh form; the loss is the mean squared error over the
first 52 outputs.
Rounded to BF16 (round to nearest even) as on the device: the weights, the
hidden activations gelu(z), the output gradient and the hidden gradients
(G W^T) * gelu'(z); sums are exact (float64) here and FP32 on the device.
"""
from __future__ import annotations

import numpy as np

IN = [64, 256, 256, 256, 256]
OUT = [256, 256, 256, 256, 64]
NO = 52


def bf16(x):
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    return (((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16).astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    """Flat parameters -> [(W [out][in], b [out])] per layer."""
    out, off = [], 0
    for i, o in zip(IN, OUT):
        W = w[off:off + o * i].reshape(o, i).astype(np.float64)
        off += o * i
        b = w[off:off + o].astype(np.float64)
        off += o
        out.append((W, b))
    return out


C_GELU = np.sqrt(2.0 / np.pi)


def gelu(z):
    """tanh form: z/2 (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3)))"""
    return 0.5 * z * (1.0 + np.tanh(C_GELU * (z + 0.044715 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(C_GELU * (z + 0.044715 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C_GELU * (1.0 + 3 * 0.044715 * z * z)


def forward(w, x):
    """x [M][64] (BF16 values) -> the network's output z [M][64] (before decoding), float64."""
    h = x.astype(np.float64)
    layers = unpack(w)
    for li, (W, b) in enumerate(layers):
        z = h @ bf16(W).T + b
        h = bf16(gelu(z)) if li < len(layers) - 1 else z
    return h


def forward_backward(w, x, t):
    """x [M][64] (BF16 values), t [M][64]; returns (loss, flat gradient)."""
    layers = unpack(w)
    M = x.shape[0]
    H, Z = [x.astype(np.float64)], []
    for li, (W, b) in enumerate(layers):
        z = H[-1] @ bf16(W).T + b
        if li < len(layers) - 1:
            Z.append(z)
            H.append(bf16(gelu(z)))
        else:
            out = z
    d = out - t
    d[:, NO:] = 0.0
    loss = float((d[:, :NO] ** 2).sum() / (M * NO))
    G = bf16(2.0 * d / (M * NO))
    grads = [None] * len(layers)
    for li in range(len(layers) - 1, -1, -1):
        W, b = layers[li]
        grads[li] = (G.T @ H[li], G.sum(axis=0))
        if li > 0:
            G = bf16((G @ bf16(W)) * gelu_grad(Z[li - 1]))
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat
