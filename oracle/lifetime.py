"""Oracle for the note-lifetime predictor (test infrastructure only).

A float64 numpy restatement of the network, loss and Adam step that the CUDA
kernels in claysampler_b200/csrc/lifetime.cu implement
(include/claysampler_lifetime.h gives the parameter layout and the loss).  The
reference has no learned part; this oracle checks the project's own kernels: the
GPU gradient against :func:`gradient`, and :func:`gradient` itself against
central finite differences (with the BF16 weight rounding switched off, since
rounding makes the loss piecewise constant in the master weights).

Also the label rule for the training renders (:func:`labels`): the peak magnitude
of a note's float render and its last frame at or above the -90 dBFS threshold.
"""
from __future__ import annotations

import numpy as np

F, H, O = 16, 64, 2
W1_AT = 0
B1_AT = W1_AT + H * F
W2_AT = B1_AT + H
B2_AT = W2_AT + H * H
W3_AT = B2_AT + H
B3_AT = W3_AT + O * H
PARAMS = B3_AT + O
NORM = 2 * F + 2 * O


def bf16(values: np.ndarray) -> np.ndarray:
    """float32 -> bfloat16 (round to nearest, ties to even), returned as float64."""
    bits = np.ascontiguousarray(values, np.float32).view(np.uint32).astype(np.uint64)
    rounded = (bits + 0x7FFF + ((bits >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params: np.ndarray, rounding: bool = True):
    p = np.asarray(params, np.float32) if rounding else np.asarray(params, np.float64)
    weight = bf16 if rounding else (lambda a: a.astype(np.float64))
    w1 = weight(p[W1_AT:B1_AT]).reshape(H, F)
    b1 = p[B1_AT:W2_AT].astype(np.float64)
    w2 = weight(p[W2_AT:B2_AT]).reshape(H, H)
    b2 = p[B2_AT:W3_AT].astype(np.float64)
    w3 = weight(p[W3_AT:B3_AT]).reshape(O, H)
    b3 = p[B3_AT:PARAMS].astype(np.float64)
    return w1, b1, w2, b2, w3, b3


def _standardise(norm: np.ndarray, features: np.ndarray) -> np.ndarray:
    norm = np.asarray(norm, np.float64)
    return (np.asarray(features, np.float64) - norm[:F]) * norm[F:2 * F]


def forward(params: np.ndarray, norm: np.ndarray, features: np.ndarray, rounding: bool = True,
            tensor: bool = True) -> np.ndarray:
    """Predictions in target units, shape (n, 2).  `tensor`: the inference kernel's
    numerics, whose first two layers run on BF16 tensor cores, so the standardised
    inputs and the first layer's activations are rounded to BF16 where they enter
    those products (cs_lifetime_forward); the training kernels keep them in FP32."""
    w1, b1, w2, b2, w3, b3 = unpack(params, rounding)
    norm = np.asarray(norm, np.float64)
    x = _standardise(norm, features)
    if tensor:
        x = bf16(x.astype(np.float32))
    h1 = np.maximum(x @ w1.T + b1, 0)
    if tensor:
        h1 = bf16(h1.astype(np.float32))
    h2 = np.maximum(h1 @ w2.T + b2, 0)
    y = h2 @ w3.T + b3
    return y * norm[2 * F + O:] + norm[2 * F:2 * F + O]


def gradient(params: np.ndarray, norm: np.ndarray, features: np.ndarray, targets: np.ndarray,
             rounding: bool = True) -> tuple[np.ndarray, float]:
    """dL/dparams (through the rounded weights) and L, for L = sum (y - t')^2 / (2n)."""
    w1, b1, w2, b2, w3, b3 = unpack(params, rounding)
    norm = np.asarray(norm, np.float64)
    x = _standardise(norm, features)
    n = x.shape[0]
    z1 = x @ w1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ w2.T + b2
    h2 = np.maximum(z2, 0)
    y = h2 @ w3.T + b3
    t = (np.asarray(targets, np.float64) - norm[2 * F:2 * F + O]) / norm[2 * F + O:]
    err = y - t
    loss = float(np.sum(err * err) / (2 * n))
    dy = err / n
    dz2 = (dy @ w3) * (z2 > 0)
    dz1 = (dz2 @ w2) * (z1 > 0)
    grad = np.zeros(PARAMS)
    grad[W1_AT:B1_AT] = (dz1.T @ x).ravel()
    grad[B1_AT:W2_AT] = dz1.sum(0)
    grad[W2_AT:B2_AT] = (dz2.T @ h1).ravel()
    grad[B2_AT:W3_AT] = dz2.sum(0)
    grad[W3_AT:B3_AT] = (dy.T @ h2).ravel()
    grad[B3_AT:PARAMS] = dy.sum(0)
    return grad, loss


def loss(params, norm, features, targets, rounding: bool = True) -> float:
    """The training loss (FP32 activations, as the training kernels compute them)."""
    y = forward(params, norm, features, rounding, tensor=False)
    norm = np.asarray(norm, np.float64)
    std = norm[2 * F + O:]
    err = (y - np.asarray(targets, np.float64)) / std
    return float(np.sum(err * err) / (2 * len(err)))


def adam(params, m, v, grad, step: int, rate: float, beta1=0.9, beta2=0.999, eps=1e-8):
    """One Adam step (returns new params, m, v)."""
    m = beta1 * m + (1 - beta1) * grad
    v = beta2 * v + (1 - beta2) * grad * grad
    mhat = m / (1 - beta1 ** step)
    vhat = v / (1 - beta2 ** step)
    return params - rate * mhat / (np.sqrt(vhat) + eps), m, v


def labels(mix: np.ndarray, windows: np.ndarray, threshold: float) -> tuple[np.ndarray, np.ndarray]:
    """Peak |sample| and last frame offset >= threshold (-1 if none) per window of a float2 mix."""
    mix = np.asarray(mix, np.float32).reshape(-1, 2)
    peaks = np.zeros(len(windows), np.float32)
    lasts = np.full(len(windows), -1, np.int32)
    for i, (first, end) in enumerate(np.asarray(windows, np.int64).reshape(-1, 2)):
        m = np.max(np.abs(mix[first:end]), axis=1) if end > first else np.zeros(0, np.float32)
        if m.size:
            peaks[i] = m.max()
            loud = np.nonzero(m >= np.float32(threshold))[0]
            if loud.size:
                lasts[i] = int(loud[-1])
    return peaks, lasts
