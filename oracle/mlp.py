"""FP64 numpy restatement of the MLP chemistry surrogate (test infrastructure).

Only the tests, the smoke check and the CPU leg of the benchmark use this
module: it is the checker of the tensor-core kernels, never the product path.
The surrogate has no counterpart in the reference, so this restates the
library's own definition (corefl-cpc_b200/csrc/surrogate.cuh):

  inputs  (12): T, ln p, bc(Y_0..Y_8), ln dt      bc(Y) = ((Y + 1e-20)^0.1 - 1)/0.1
  outputs (11): bc(Y_new) - bc(Y_old), dT, ln(reaction time scale), each learnt
                as asinh(g / scale) (g itself for a zero scale), standardised
  network: 16 -> 128 tanh -> 128 tanh -> 128 tanh -> 16, biases folded in as
  constant-1 columns (input column 15; hidden column 128 of 144).
  loss: mean over rows and the 11 outputs of the squared standardised error.

`bf16=True` rounds what the kernels round (weights, the standardised inputs,
every activation tile, the output gradient and every dz tile) to bfloat16,
nearest-even, while accumulating in FP64; the kernels accumulate in FP32 and
use the hardware tanh approximation, so they agree with that variant to a few
BF16 ulps and with the plain FP64 variant to the BF16 rounding level.
"""
from __future__ import annotations

import numpy as np

NIN, NOUT, H, KH = 12, 11, 128, 144
OFF = (0, 128 * 16, 128 * 16 + 128 * 144, 128 * 16 + 2 * 128 * 144)
SHAPES = ((128, 16), (128, 144), (128, 144), (16, 144))
NPARAM = OFF[3] + 16 * 144
LAMBDA, EPS = 0.1, 1e-20


def bf16(x) -> np.ndarray:
    """Round to bfloat16 (nearest even), returned as float64."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32)
    r = ((a + np.uint32(0x7FFF) + ((a >> np.uint32(16)) & np.uint32(1))) & np.uint32(0xFFFF0000)).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def unpack(w):
    w = np.asarray(w, dtype=np.float64)
    return [w[OFF[b]:OFF[b] + SHAPES[b][0] * SHAPES[b][1]].reshape(SHAPES[b]) for b in range(4)]


def pack(blocks) -> np.ndarray:
    return np.concatenate([np.asarray(b, dtype=np.float64).ravel() for b in blocks])


def boxcox(y):
    return ((np.maximum(y, 0.0) + EPS) ** LAMBDA - 1.0) / LAMBDA


def boxcox_inv(b):
    x = 1.0 + LAMBDA * np.asarray(b, dtype=np.float64)
    return np.where(x > 0, np.maximum(np.maximum(x, 0) ** 10 - EPS, 0.0), 0.0)


def raw_features(T, p, Y, dt):
    """Rows of the 12 raw inputs; Y is (n, ns) with ns <= 9."""
    T = np.atleast_1d(np.asarray(T, dtype=np.float64))
    n = T.shape[0]
    f = np.zeros((n, NIN))
    f[:, 0] = T
    f[:, 1] = np.log(np.broadcast_to(p, (n,)))
    Y = np.atleast_2d(Y)
    f[:, 2:2 + Y.shape[1]] = boxcox(Y)
    f[:, 11] = np.log(np.broadcast_to(dt, (n,)))
    return f


def standardise_inputs(X, norm):
    nm = split_norm(norm)
    return (np.asarray(X, np.float64) - nm["in_mean"]) * nm["in_rstd"]


def standardise_targets(G, norm):
    nm = split_norm(norm)
    sc = nm["out_scale"]
    G = np.asarray(G, np.float64)
    z = np.where(sc > 0, np.arcsinh(G / np.where(sc > 0, sc, 1.0)), G)
    return (z - nm["out_mean"]) / nm["out_std"]


def destandardise_outputs(Y, norm):
    """Network outputs (standardised learnt variables) -> raw increments."""
    nm = split_norm(norm)
    sc = nm["out_scale"]
    z = nm["out_mean"] + nm["out_std"] * np.asarray(Y, np.float64)[:, :NOUT]
    return np.where(sc > 0, sc * np.sinh(z), z)


def split_norm(norm):
    v = np.asarray(norm, dtype=np.float64)
    return {"in_mean": v[0:12], "in_rstd": v[12:24], "out_mean": v[24:35], "out_std": v[35:46],
            "in_lo": v[46:58], "in_hi": v[58:70], "out_scale": v[70:81]}


def forward(w, Xs, bf16_round=False):
    """Standardised inputs (n, 12) -> (outputs (n, 16), activations a0..a3)."""
    r = bf16 if bf16_round else (lambda v: np.asarray(v, dtype=np.float64))
    W = [r(b) for b in unpack(w)]
    n = Xs.shape[0]
    a0 = np.zeros((n, 16))
    a0[:, :NIN] = Xs
    a0 = r(a0)
    a0[:, 15] = 1.0
    acts = [a0]
    a = a0
    for l in range(3):
        h = np.tanh(a @ W[l].T)
        nxt = np.zeros((n, KH))
        nxt[:, :H] = r(h)
        nxt[:, H] = 1.0
        acts.append(nxt)
        a = nxt
    y = a @ W[3].T
    return y, acts


def loss_and_grad(w, Xs, Ts, bf16_round=False):
    """Mean squared standardised error over the 11 outputs and its gradient
    with respect to the flat parameter vector (layout of the library)."""
    r = bf16 if bf16_round else (lambda v: np.asarray(v, dtype=np.float64))
    W = [r(b) for b in unpack(w)]
    y, acts = forward(w, Xs, bf16_round)
    n = Xs.shape[0]
    e = np.zeros((n, 16))
    e[:, :NOUT] = y[:, :NOUT] - Ts
    loss = float((e ** 2).sum() / (n * NOUT))
    dy = e * (2.0 / (n * NOUT))
    g3 = np.zeros((16, KH))
    dyr = r(dy)
    g3[:, :H] = dyr.T @ acts[3][:, :H]
    g3[:, H] = dy.sum(axis=0)  # bias gradient from the unrounded dy
    grads = [None, None, None, g3]
    dz = dyr
    for l in (3, 2, 1):
        dh = dz @ W[l][:, :H]
        hl = acts[l][:, :H]
        dzl = r(dh * (1.0 - hl * hl))
        g = dzl.T @ acts[l - 1]
        grads[l - 1] = g
        dz = dzl
    return loss, pack(grads)


def init_weights(seed=0):
    """Xavier-uniform weights, zero biases (numpy generator; for CPU tests)."""
    rng = np.random.default_rng(seed)
    blocks = []
    for b, (rows, cols) in enumerate(SHAPES):
        fan_in = NIN if b == 0 else H
        fan_out = NOUT if b == 3 else H
        lim = np.sqrt(6.0 / (fan_in + fan_out))
        m = np.zeros((rows, cols))
        m[:fan_out, :fan_in] = rng.uniform(-lim, lim, (fan_out, fan_in))
        blocks.append(m)
    return pack(blocks)
