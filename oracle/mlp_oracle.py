"""TEST INFRASTRUCTURE: CPU FP64 restatement of the surrogate network's
forward and backward passes (bes_mlp_forward / bes_mlp_backward).

It rounds at the same places the CUDA kernels do (inputs after
standardisation and hidden activations to BF16, weights to BF16 for the
products, biases in FP32) and then computes everything else in FP64, so the
kernels' FP32 accumulation is the only difference left.  Only the tests use it.
"""
from __future__ import annotations

import numpy as np

C_GELU = 0.7978845608028654


def f32(x) -> np.ndarray:
    """Round to FP32 (the kernels' master weights, inputs and statistics are FP32)."""
    return np.asarray(np.asarray(x, np.float64).astype(np.float32), np.float64)


def bf16(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (nearest, ties to even), returned as float64."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    t = np.tanh(C_GELU * (x + 0.044715 * x ** 3))
    return 0.5 * x * (1.0 + t)


def gelu_d(x):
    t = np.tanh(C_GELU * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * C_GELU * (1.0 + 3.0 * 0.044715 * x * x)


def unpack(params: np.ndarray, sizes):
    """sizes: list of (fan_in, fan_out); returns [(W [out][in], b [out])]."""
    out, k = [], 0
    for fi, fo in sizes:
        W = params[k:k + fi * fo].reshape(fo, fi).astype(np.float64)
        k += fi * fo
        b = params[k:k + fo].astype(np.float64)
        k += fo
        out.append((W, b))
    assert k == params.size
    return out


def layer_sizes(n_in, width, depth, n_out):
    return [(n_in if l == 0 else width, n_out if l == depth else width) for l in range(depth + 1)]


def forward(params, sizes, x, in_mean, in_std, out_mean, out_std):
    layers = unpack(params, sizes)
    a = bf16(f32((f32(x) - f32(in_mean)) / f32(in_std)))
    acts, pres = [a], []
    for l, (W, b) in enumerate(layers):
        z = a @ bf16(f32(W)).T + f32(b)
        pres.append(z)
        if l + 1 < len(layers):
            a = bf16(f32(gelu(z)))
            acts.append(a)
    y = pres[-1] * np.asarray(out_std, np.float64) + np.asarray(out_mean, np.float64)
    return y, acts, pres


def backward(params, sizes, x, t, in_mean, in_std, out_mean, out_std):
    """Loss (mean squared error of standardised outputs) and its gradient, same layout as params."""
    layers = unpack(params, sizes)
    _, acts, pres = forward(params, sizes, x, in_mean, in_std, out_mean, out_std)
    B, n_out = pres[-1].shape
    tn = (np.asarray(t, np.float64) - np.asarray(out_mean, np.float64)) / np.asarray(out_std, np.float64)
    d = pres[-1] - tn
    loss = float((d * d).mean())
    dz = 2.0 * d / (B * n_out)
    grads = [None] * len(layers)
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        gW = dz.T @ acts[l]
        gb = dz.sum(0)
        grads[l] = (gW, gb)
        if l > 0:
            dx = dz @ bf16(f32(W))
            dz = dx * gelu_d(pres[l - 1])
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return loss, flat
