"""Test infrastructure only: a CPU restatement of the learned warm start's network (beamlab_b200/csrc/bl_mlp.cuh,
which has no counterpart in the reference) - the checker of the GPU's forward and gradient kernels.

36 -> 64 -> 64 -> 64 -> 12, ReLU, the parameters in one vector (W1 64x36 row = output, b1, W2 64x64, b2, W3 64x64,
b3, W4 12x64, b4), the forward on the BF16-rounded parameters and BF16-rounded layer inputs (as the GPU's tensor cores
take them), accumulation in float64 here.
Loss over n samples: sum_s sum_o w_so (y_so - t_so)^2 / (2 n).
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 36, 64, 12
SHAPES = [("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
          ("W3", (N_HID, N_HID)), ("b3", (N_HID,)), ("W4", (N_OUT, N_HID)), ("b4", (N_OUT,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16(x: np.ndarray) -> np.ndarray:
    """float32 -> the nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray) -> dict:
    out, o = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = p[o:o + k].reshape(shape)
        o += k
    return out


def forward(p: np.ndarray, x: np.ndarray, round_bf16: bool = True):
    """Outputs and activations of the network on samples x (n x 36), in float64. round_bf16: the parameters and each
    layer's input rounded to BF16, as the GPU's tensor cores take them (the activations returned are those inputs)."""
    q = unpack((bf16(p) if round_bf16 else p).astype(np.float64))
    rnd = (lambda a: bf16(np.asarray(a, np.float32)).astype(np.float64)) if round_bf16 else (lambda a: np.asarray(a, np.float64))
    a0 = rnd(x)
    z1 = a0 @ q["W1"].T + q["b1"]
    a1 = rnd(np.maximum(z1, 0))
    z2 = a1 @ q["W2"].T + q["b2"]
    a2 = rnd(np.maximum(z2, 0))
    z3 = a2 @ q["W3"].T + q["b3"]
    a3 = rnd(np.maximum(z3, 0))
    y = a3 @ q["W4"].T + q["b4"]
    return y, (a0, a1, a2, a3)


def loss_and_grad(p: np.ndarray, x: np.ndarray, t: np.ndarray, w: np.ndarray, round_bf16: bool = True):
    """(loss, gradient) of the loss with respect to the parameters the forward uses."""
    n = len(x)
    y, (a0, a1, a2, a3) = forward(p, x, round_bf16)
    q = unpack((bf16(p) if round_bf16 else p).astype(np.float64))
    e = y - t
    loss = 0.5 * np.sum(w * e * e) / n
    d4 = w * e / n
    g = {"W4": d4.T @ a3, "b4": d4.sum(0)}
    d3 = (d4 @ q["W4"]) * (a3 > 0)
    g["W3"], g["b3"] = d3.T @ a2, d3.sum(0)
    d2 = (d3 @ q["W3"]) * (a2 > 0)
    g["W2"], g["b2"] = d2.T @ a1, d2.sum(0)
    d1 = (d2 @ q["W2"]) * (a1 > 0)
    g["W1"], g["b1"] = d1.T @ a0, d1.sum(0)
    return loss, np.concatenate([g[name].ravel() for name, _ in SHAPES])


def central_difference(p: np.ndarray, x, t, w, indices, h=1e-6):
    """The loss's derivative by central differences at the given parameter indices (float64, no rounding)."""
    p = np.asarray(p, np.float64)
    out = []
    for i in indices:
        a, b = p.copy(), p.copy()
        a[i] += h
        b[i] -= h
        out.append((loss_and_grad(a, x, t, w, False)[0] - loss_and_grad(b, x, t, w, False)[0]) / (2 * h))
    return np.asarray(out)
