"""CPU restatement of the learned k-proposal network (test infrastructure only).

The product trains and runs the network with its own CUDA kernels (apo_b200/csrc/proposal.cu);
this module recomputes the same forward pass, loss and gradients in float64 numpy from the same
bf16-rounded weights, so the tests can check the GPU's gradients (and predictions) against it.
The reference has no such network: it only measures, per kNN rank, whether a neighbour
contributed and whether the security radius was reached
(app/benchmarks/benchmark_contributing_nearest.cu:10-129), which is where the training labels
come from.

Network: 16 -> 64 -> 64 -> 1, ReLU, weights stored in bf16 (rounded to nearest even from the
fp32 master copy), biases fp32, fp32 accumulation on the GPU. Inputs are normalised as
(x - mean) * inv_scale before the first layer. Loss: mean squared error on log2 of the
certified rank. Parameter vector order: W1 (64 x 16, row-major), b1 (64), W2 (64 x 64), b2 (64),
w3 (64), b3 (1): 5,313 values.
"""
from __future__ import annotations

import numpy as np

IN, HID = 16, 64
SHAPES = [("w1", (HID, IN)), ("b1", (HID,)), ("w2", (HID, HID)), ("b2", (HID,)), ("w3", (HID,)), ("b3", (1,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)
WEIGHTS = ("w1", "w2", "w3")


def bf16_round(a: np.ndarray) -> np.ndarray:
    """fp32 -> bf16 (round to nearest even) -> fp32, as __float2bfloat16_rn does."""
    x = np.ascontiguousarray(a, dtype=np.float32)
    bits = x.view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    out = rounded.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(x), x, out)


def unpack(params: np.ndarray) -> dict:
    out, at = {}, 0
    for name, shape in SHAPES:
        size = int(np.prod(shape))
        out[name] = np.asarray(params[at:at + size], dtype=np.float64).reshape(shape)
        at += size
    return out


def pack(parts: dict) -> np.ndarray:
    return np.concatenate([np.asarray(parts[name], dtype=np.float64).reshape(-1) for name, _ in SHAPES])


def effective(params: np.ndarray) -> dict:
    """The parameters the forward pass uses: weights rounded to bf16, biases as they are."""
    p = unpack(np.asarray(params, dtype=np.float32))
    for name in WEIGHTS:
        p[name] = bf16_round(p[name].astype(np.float32)).astype(np.float64)
    return p


def normalise(x: np.ndarray, mean: np.ndarray, inv_scale: np.ndarray) -> np.ndarray:
    return (np.asarray(x, np.float64) - np.asarray(mean, np.float64)) * np.asarray(inv_scale, np.float64)


def forward(params: np.ndarray, xn: np.ndarray):
    p = effective(params)
    z1 = xn @ p["w1"].T + p["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ p["w2"].T + p["b2"]
    h2 = np.maximum(z2, 0.0)
    o = h2 @ p["w3"] + p["b3"][0]
    return o, (h1, h2, p)


def loss_and_gradients(params: np.ndarray, xn: np.ndarray, y: np.ndarray):
    """Mean squared error and its gradient with respect to every parameter (the gradient
    of the bf16 weights is taken as the gradient of their fp32 masters)."""
    o, (h1, h2, p) = forward(params, xn)
    b = xn.shape[0]
    r = o - np.asarray(y, np.float64)
    loss = float(np.mean(r * r))
    g = 2.0 * r / b
    grads = {"w3": h2.T @ g, "b3": np.array([g.sum()])}
    d2 = np.outer(g, p["w3"]) * (h2 > 0)
    grads["w2"] = d2.T @ h1
    grads["b2"] = d2.sum(axis=0)
    d1 = (d2 @ p["w2"]) * (h1 > 0)
    grads["w1"] = d1.T @ xn
    grads["b1"] = d1.sum(axis=0)
    return loss, pack(grads)


def finite_difference(params: np.ndarray, xn: np.ndarray, y: np.ndarray, index: int, h: float = 1e-3) -> float:
    """Central difference of the loss in one parameter, with the forward pass in float64 and
    no bf16 rounding (checks the analytic gradient formulas themselves)."""
    def loss_at(pv):
        p = unpack(pv)
        h1 = np.maximum(xn @ p["w1"].T + p["b1"], 0.0)
        h2 = np.maximum(h1 @ p["w2"].T + p["b2"], 0.0)
        o = h2 @ p["w3"] + p["b3"][0]
        return float(np.mean((o - y) ** 2))
    up = np.array(params, dtype=np.float64)
    dn = np.array(params, dtype=np.float64)
    up[index] += h
    dn[index] -= h
    return (loss_at(up) - loss_at(dn)) / (2 * h)


def analytic_float64(params: np.ndarray, xn: np.ndarray, y: np.ndarray) -> np.ndarray:
    """Gradient formulas of loss_and_gradients without bf16 rounding (for finite_difference)."""
    p = unpack(np.asarray(params, dtype=np.float64))
    h1 = np.maximum(xn @ p["w1"].T + p["b1"], 0.0)
    h2 = np.maximum(h1 @ p["w2"].T + p["b2"], 0.0)
    o = h2 @ p["w3"] + p["b3"][0]
    g = 2.0 * (o - y) / xn.shape[0]
    d2 = np.outer(g, p["w3"]) * (h2 > 0)
    d1 = (d2 @ p["w2"]) * (h1 > 0)
    return pack({"w1": d1.T @ xn, "b1": d1.sum(axis=0), "w2": d2.T @ h1, "b2": d2.sum(axis=0),
                 "w3": h2.T @ g, "b3": np.array([g.sum()])})
