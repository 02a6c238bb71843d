"""CPU oracle of the learned-correction network -- TEST INFRASTRUCTURE ONLY.

A float64 numpy statement of the network the library trains on the GPU (the network has no
counterpart in the reference: it is the learned part of the task, configuration 4): five 3x3
convolutions with zero padding, 4 -> 32 -> 32 -> 32 -> 32 -> 4 channels, GELU (x * Phi(x))
between them, the mean-squared-error loss of the normalised correction, and the gradients of
every parameter by backpropagation.  The GPU keeps activations, weights and output gradients in
bfloat16; this oracle rounds the same quantities to bfloat16 at the same points (round to
nearest even), so the remaining differences are the order of FP32 accumulation and float32
pre-activations.  Parameters use the library's padded layout: per layer weights
[cout_p][9][cin_p] (tap t = 3 * dy + dx, offsets dy - 1, dx - 1) then biases [cout_p], with
cin_p = 16, 32, 32, 32, 32 and cout_p = 32, 32, 32, 32, 8.

Only the tests import this module.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

CIN_P = (16, 32, 32, 32, 32)
COUT_P = (32, 32, 32, 32, 8)
IMG = 64


def bf16(a):
    """Round float values to bfloat16 (nearest even) and return them as float64."""
    f = np.asarray(a, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def unpack(params):
    """Split the flat parameter vector into [(W[cout][9][cin], b[cout]), ...]."""
    out, off = [], 0
    for ci, co in zip(CIN_P, COUT_P):
        w = np.asarray(params[off:off + co * 9 * ci], dtype=np.float64).reshape(co, 9, ci)
        off += co * 9 * ci
        b = np.asarray(params[off:off + co], dtype=np.float64)
        off += co
        out.append((w, b))
    return out


def pack(layers):
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in layers])


def patches(x):
    """x [n][64][64][c] -> [n*4096][9*c]: the 9 zero-padded neighbours of every pixel, tap-major."""
    n, h, w, c = x.shape
    xp = np.zeros((n, h + 2, w + 2, c))
    xp[:, 1:-1, 1:-1] = x
    cols = [xp[:, dy:dy + h, dx:dx + w] for dy in range(3) for dx in range(3)]
    return np.stack(cols, axis=3).reshape(n * h * w, 9 * c)


def conv(x, w):
    """3x3 convolution: out[p][co] = sum_t sum_k x[p + off(t)][k] w[co][t][k]."""
    n = x.shape[0]
    co = w.shape[0]
    return (patches(x) @ w.reshape(co, -1).T).reshape(n, IMG, IMG, co)


def conv_input_grad(dz, w):
    """Adjoint of conv with respect to its input: g[p][k] = sum_t sum_co dz[p - off(t)][co] w[co][t][k]."""
    wf = w[:, ::-1, :].transpose(2, 1, 0)  # [k][t'][co] with t' = 8 - t
    return conv(dz, wf)


def conv_weight_grad(x, dz):
    """dW[co][t][k] = sum_p dz[p][co] x[p + off(t)][k]."""
    n = x.shape[0]
    pt = patches(x)  # [P][9*cin]
    g = dz.reshape(n * IMG * IMG, -1).T @ pt  # [co][9*cin]
    return g.reshape(dz.shape[-1], 9, x.shape[-1])


def input_tensor(coarse, in_mean, in_scale):
    """coarse [n][4][64][64] -> normalised bf16 input [n][64][64][16]."""
    n = coarse.shape[0]
    a = np.zeros((n, IMG, IMG, 16))
    for c in range(4):
        a[..., c] = (np.asarray(coarse[:, c], dtype=np.float32) - np.float32(in_mean[c])) * np.float32(1.0 / in_scale[c])
    return bf16(a)


def forward(params, coarse, in_mean, in_scale):
    """Network output y [n][64][64][8] (channels 0..3 used) and the intermediate values."""
    layers = unpack(params)
    a = [input_tensor(coarse, in_mean, in_scale)]
    z = []
    for l, (w, b) in enumerate(layers):
        out = conv(a[l], bf16(w)) + np.asarray(b, dtype=np.float32)
        if l < 4:
            z.append(out)
            a.append(bf16(gelu(out)))
        else:
            y = out
    return y, a, z


def loss_and_grads(params, coarse, fine_r, in_mean, in_scale, out_scale):
    """Loss (mean squared error of y[..., :4] against (fine_r - coarse) / out_scale) and the
    gradient of every parameter, in the library's flat layout."""
    layers = unpack(params)
    y, a, z = forward(params, coarse, in_mean, in_scale)
    n = coarse.shape[0]
    t = np.stack([(fine_r[:, c] - coarse[:, c]) / out_scale[c] for c in range(4)], axis=-1)
    d = y[..., :4] - t
    count = d.size
    loss = float(np.sum(d * d) / count)
    dz = np.zeros((n, IMG, IMG, 16))
    dz[..., :4] = bf16(2.0 * d / count)
    grads = [None] * 5
    for l in range(4, -1, -1):
        w, _ = layers[l]
        co = w.shape[0]
        dzl = dz[..., :co]
        gw = conv_weight_grad(a[l], dzl)
        gb = dzl.sum(axis=(0, 1, 2))
        grads[l] = (gw, gb)
        if l > 0:
            da = conv_input_grad(dzl, bf16(w))
            dz = bf16(da * gelu_grad(z[l - 1]))
    return loss, pack(grads)
