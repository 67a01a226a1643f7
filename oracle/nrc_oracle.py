"""CPU restatement of the neural radiance cache's network (TEST INFRASTRUCTURE
ONLY: tests/ use it as the checker of the sm_100a MLP kernels; nothing in the
product imports it).

The radiance cache has no counterpart in the reference, so this module is the
specification the GPU kernels are checked against.  It follows the kernels'
mixed precision step by step:

  encode   96 inputs per sample, rounded to bf16 (round to nearest even):
             [ 0,72)  position p (scene box mapped to [0,1]^3), per axis c and
                      octave k = 0..11: sin(2^k pi p_c), cos(2^k pi p_c)  (index 24c+2k, +1)
             [72,88)  direction: real spherical harmonics of bands 0..3
             [88,91)  shading normal      [91] roughness
             [92,95)  albedo              [95] constant 1 (the first layer's bias)
  forward  four hidden layers of 64 ReLU units, no biases past the first:
             H_{l+1} = bf16(relu(H_l W_l^T))  with f32 accumulation,
           output z = H_4 W_4^T (3 channels), radiance = max(exp(min(z, 15)) - 0.01, 0)
  loss     L2 in log space: (z - log(y + 0.01))^2, averaged over samples and
           channels (z regresses log radiance; the gradient through an exp
           output never vanishes, unlike a relative L2 on exp(z))
  backward per-sample output gradient dz = 2 (z - log(y + 0.01)), rounded to
           bf16; hidden gradients
           g_l = bf16(dH_l * [H_l > 0]),  dH_l = g_{l+1} W_l  (f32 accumulation);
           weight gradients dW_l = sum over samples of g^T H, divided by 3 * batch
  adam     Kingma & Ba 2015 with bias correction; the f32 master weights are
           the state, the kernels read their bf16 rounding.

Parameters are one flat float32 vector: W0 [64][96], W1..W3 [64][64], W4 [3][64]
(row = output unit).
"""
from __future__ import annotations

import numpy as np

N_IN, N_HIDDEN, N_OUT = 96, 64, 3
SHAPES = [(64, 96), (64, 64), (64, 64), (64, 64), (3, 64)]
N_PARAMS = sum(a * b for a, b in SHAPES)
OCTAVES = 12
LOG_OFFSET = 0.01
Z_MAX = 15.0


def bf16(x):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float32."""
    a = np.ascontiguousarray(np.asarray(x, np.float32))
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(a.shape)


def unpack(params, dtype=np.float32):
    out, o = [], 0
    for r, c in SHAPES:
        out.append(np.asarray(params[o:o + r * c], dtype).reshape(r, c))
        o += r * c
    return out


def pack(mats):
    return np.concatenate([np.asarray(m, np.float32).ravel() for m in mats])


def sh_bands4(d):
    """Real spherical harmonics of bands 0..3 (16 values) of unit vectors d [n,3]."""
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz = x * x, y * y, z * z
    return np.stack([
        np.full_like(x, 0.28209479177387814),
        -0.48860251190291987 * y,
        0.48860251190291987 * z,
        -0.48860251190291987 * x,
        1.0925484305920792 * x * y,
        -1.0925484305920792 * y * z,
        0.94617469575755997 * zz - 0.31539156525251999,
        -1.0925484305920792 * x * z,
        0.54627421529603959 * (xx - yy),
        0.59004358992664352 * y * (3 * xx - yy) * -1.0,
        2.8906114426405538 * x * y * z,
        0.45704579946446572 * y * (1 - 5 * zz),
        0.3731763325901154 * z * (5 * zz - 3),
        0.45704579946446572 * x * (1 - 5 * zz),
        1.4453057213202769 * z * (xx - yy),
        0.59004358992664352 * x * (3 * yy - xx),
    ], axis=1)


def encode(features):
    """features [n,16] float32: (p.xyz, roughness) (dir.xyz, 0) (normal.xyz, 0) (albedo.xyz, 0)."""
    f = np.asarray(features, np.float32).reshape(-1, 16)
    n = len(f)
    X = np.zeros((n, N_IN), np.float64)
    p = f[:, 0:3].astype(np.float64)
    for c in range(3):
        for k in range(OCTAVES):
            a = np.float32(2.0 ** k) * f[:, c]          # exact in float32
            X[:, 24 * c + 2 * k] = np.sin(np.pi * a.astype(np.float64))
            X[:, 24 * c + 2 * k + 1] = np.cos(np.pi * a.astype(np.float64))
    X[:, 72:88] = sh_bands4(f[:, 4:7].astype(np.float64))
    X[:, 88:91] = f[:, 8:11]
    X[:, 91] = f[:, 3]
    X[:, 92:95] = f[:, 12:15]
    X[:, 95] = 1.0
    del p
    return bf16(X.astype(np.float32))


def _round(x, rounding):
    return bf16(np.asarray(x, np.float32)).astype(np.float64) if rounding else np.asarray(x, np.float64)


def forward(params, X, rounding=True):
    """rounding=False: the same network in float64 throughout (for derivative checks)."""
    W = [_round(w, True) for w in unpack(params)] if rounding else unpack(params, np.float64)
    H = [np.asarray(X, np.float64)]
    for l in range(4):
        H.append(_round(np.maximum(H[-1] @ W[l].T, 0.0), rounding))
    z = H[-1] @ W[4].T
    y = np.maximum(np.exp(np.minimum(z, Z_MAX)) - LOG_OFFSET, 0.0)
    return {"H": H, "z": z, "y": y, "W": W}


def infer(params, features):
    return forward(params, encode(features))["y"].astype(np.float32)


def loss_and_output_gradient(fw, target):
    z = fw["z"]
    t = np.log(np.maximum(np.asarray(target, np.float64)[:, :3], 0.0) + LOG_OFFSET)
    diff = z - t
    return float(np.mean(diff * diff)), 2.0 * diff


def gradients(params, features, target, rounding=True, X=None):
    """Mean-loss gradient (flat, like params) and the loss, as the kernels compute them
    (rounding=False: exact float64 derivatives of the unrounded network)."""
    fw = forward(params, encode(features) if X is None else X, rounding)
    loss, dz = loss_and_output_gradient(fw, target)
    H, W = fw["H"], fw["W"]
    n = len(dz)
    g = _round(dz, rounding)
    grads = [None] * 5
    grads[4] = g.T @ H[4]
    for l in range(3, -1, -1):
        dH = g @ W[l + 1]
        g = _round(dH * (H[l + 1] > 0), rounding)
        grads[l] = g.T @ H[l]
    scale = 1.0 / (3.0 * n)
    return pack([gr * scale for gr in grads]), loss


def adam(params, m, v, grad, step, lr=1e-2, beta1=0.9, beta2=0.99, eps=1e-8):
    """One Adam update (step counts from 1); returns new (params, m, v) as float32."""
    p = np.asarray(params, np.float64)
    m = beta1 * np.asarray(m, np.float64) + (1 - beta1) * grad
    v = beta2 * np.asarray(v, np.float64) + (1 - beta2) * grad * grad
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    p = p - lr * mh / (np.sqrt(vh) + eps)
    return p.astype(np.float32), m.astype(np.float32), v.astype(np.float32)
