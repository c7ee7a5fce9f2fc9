"""Test infrastructure, not product code: a float64 NumPy restatement of the guiding
network (encoding -> MLP -> von Mises-Fisher mixture -> loss gradient -> Adam).

Pine has no path guiding, so this oracle restates the specification the GPU kernels
implement (pine_b200/csrc/guide_net.cuh, guide_mlp.cu) rather than a reference
implementation; it is checked against itself by finite differences in tests/.

Only tests/ use this module.
"""

from __future__ import annotations

import numpy as np

FEATURES = 32
DIM = 64
LAYERS = 6
LOBES = 8
OUTPUTS = 40
BINS = 5
LOG_KAPPA_MIN, LOG_KAPPA_MAX = -3.0, 7.0
GRAD_CLIP = 1.0e4


# ---------------------------------------------------------------- encoding
def one_blob(x):
    c = (np.arange(BINS) + 0.5) / BINS
    d = (x[:, None] - c[None, :]) * BINS
    return np.exp(-0.5 * d * d)


def angles(d):
    t = np.arccos(np.clip(d[:, 2], -1.0, 1.0)) / np.pi
    p = np.arctan2(d[:, 1], d[:, 0])
    p = np.where(p < 0, p + 2 * np.pi, p) / (2 * np.pi)
    return t, p


def encode(pos_unit, normal, wo):
    """Features (n x 32); a NaN normal x marks a medium vertex (normal features 0)."""
    pos_unit = np.asarray(pos_unit, np.float64)
    normal = np.asarray(normal, np.float64)
    wo = np.asarray(wo, np.float64)
    n = pos_unit.shape[0]
    f = np.zeros((n, FEATURES))
    x = np.clip(pos_unit, 0.0, 1.0)
    for a in range(3):
        for k in range(2):
            w = np.pi * (1 << k) * x[:, a]
            f[:, 4 * a + 2 * k] = np.sin(w)
            f[:, 4 * a + 2 * k + 1] = np.cos(w)
    has = ~np.isnan(normal[:, 0])
    nn = np.where(has[:, None], normal, 0.0)
    t, p = angles(nn)
    f[:, 12:17] = np.where(has[:, None], one_blob(t), 0.0)
    f[:, 17:22] = np.where(has[:, None], one_blob(p), 0.0)
    t, p = angles(wo)
    f[:, 22:27] = one_blob(t)
    f[:, 27:32] = one_blob(p)
    return f


def input_rows(features):
    """Feature rows padded to the network's 64 inputs with the constant input 32."""
    n = features.shape[0]
    x = np.zeros((n, DIM))
    x[:, :FEATURES] = features
    x[:, FEATURES] = 1.0
    return x


# ---------------------------------------------------------------- vMF mixture
def log_norm(kappa):
    return np.log(kappa) - np.log(2 * np.pi) - np.log1p(-np.exp(-2 * kappa))


def mixture(raw):
    """(mu n x 8 x 3, kappa n x 8, weight n x 8) of raw outputs (n x 40)."""
    r = np.asarray(raw, np.float64).reshape(-1, LOBES, 5)
    v = r[:, :, :3]
    ln = np.linalg.norm(v, axis=2, keepdims=True)
    mu = np.where(ln > 1e-20, v / np.maximum(ln, 1e-300), np.array([0.0, 0.0, 1.0]))
    kappa = np.exp(np.clip(r[:, :, 3], LOG_KAPPA_MIN, LOG_KAPPA_MAX))
    a = r[:, :, 4]
    w = np.exp(a - a.max(axis=1, keepdims=True))
    w /= w.sum(axis=1, keepdims=True)
    return mu, kappa, w


def pdf(raw, dirs):
    mu, kappa, w = mixture(raw)
    c = np.einsum("nkj,nj->nk", mu, np.asarray(dirs, np.float64))
    return (w * np.exp(log_norm(kappa) + kappa * (c - 1.0))).sum(axis=1)


def loss_and_grad(raw, dir_weight):
    """Per-sample -w log q(d) and its gradient with respect to the raw outputs."""
    raw = np.asarray(raw, np.float64)
    dw = np.asarray(dir_weight, np.float64)
    r = raw.reshape(-1, LOBES, 5)
    d, wt = dw[:, :3], dw[:, 3]
    v = r[:, :, :3]
    ln = np.linalg.norm(v, axis=2)
    mu = v / np.maximum(ln, 1e-300)[:, :, None]
    lk = r[:, :, 3]
    kappa = np.exp(np.clip(lk, LOG_KAPPA_MIN, LOG_KAPPA_MAX))
    c = np.einsum("nkj,nj->nk", mu, d)
    a = r[:, :, 4]
    logw = a - (a.max(axis=1, keepdims=True) +
                np.log(np.exp(a - a.max(axis=1, keepdims=True)).sum(axis=1, keepdims=True)))
    logp = log_norm(kappa) + kappa * (c - 1.0)
    t = logw + logp
    lq = t.max(axis=1) + np.log(np.exp(t - t.max(axis=1, keepdims=True)).sum(axis=1))
    resp = np.exp(t - lq[:, None])
    g = -wt[:, None]
    grad = np.zeros_like(r)
    grad[:, :, 4] = g * (resp - np.exp(logw))
    free = (lk > LOG_KAPPA_MIN) & (lk < LOG_KAPPA_MAX)
    with np.errstate(over="ignore"):  # expm1 overflows to inf for large kappa: term 0
        dlk = 1.0 / kappa - 2.0 / np.expm1(2.0 * kappa) + (c - 1.0)
    grad[:, :, 3] = np.where(free, g * resp * kappa * dlk, 0.0)
    s = g * resp * kappa / ln
    grad[:, :, :3] = (d[:, None, :] - mu * c[:, :, None]) * s[:, :, None]
    return -wt * lq, grad.reshape(-1, OUTPUTS)


def sample(raw, u):
    """Directions drawn with uniforms u (n x 3): lobe by weight, vMF cosine by inverting
    its CDF, uniform azimuth."""
    mu, kappa, w = mixture(raw)
    u = np.asarray(u, np.float64)
    cdf = np.cumsum(w, axis=1)
    k = np.minimum((u[:, :1] >= cdf).sum(axis=1), LOBES - 1)
    idx = np.arange(len(k))
    m, kap = mu[idx, k], kappa[idx, k]
    uu = np.maximum(u[:, 1], 1e-7)
    c = np.clip(1.0 + np.log(uu + (1.0 - uu) * np.exp(-2.0 * kap)) / kap, -1.0, 1.0)
    s = np.sqrt(np.maximum(0.0, 1.0 - c * c))
    phi = 2 * np.pi * u[:, 2]
    sg = np.where(m[:, 2] >= 0, 1.0, -1.0)
    a = -1.0 / (sg + m[:, 2])
    b = m[:, 0] * m[:, 1] * a
    b1 = np.stack([1.0 + sg * m[:, 0] ** 2 * a, sg * b, -sg * m[:, 0]], axis=1)
    b2 = np.stack([b, sg + m[:, 1] ** 2 * a, -m[:, 1]], axis=1)
    return (b1 * (s * np.cos(phi))[:, None] + b2 * (s * np.sin(phi))[:, None] +
            m * c[:, None])


# ---------------------------------------------------------------- network
def _h(x, fp16):
    return x.astype(np.float16).astype(np.float64) if fp16 else x


def forward(weights, features, fp16=True):
    """Raw outputs and every layer's input.  With fp16 the weights, inputs and activations
    are rounded to FP16 as the tensor-core kernels store them; sums stay float64."""
    W = [_h(np.asarray(weights, np.float64)[l], fp16) for l in range(LAYERS)]
    h = _h(input_rows(np.asarray(features, np.float64)), fp16)
    acts = [h]
    for l in range(LAYERS):
        z = h @ W[l].T
        if l + 1 < LAYERS:
            h = _h(np.maximum(z, 0.0), fp16)
            acts.append(h)
    return z[:, :OUTPUTS], acts


def gradient(weights, features, dir_weight, weight_scale=1.0, fp16=True):
    """Mean gradient (6 x 64 x 64) of -w log q(d) over the samples and the mean loss,
    with the kernels' per-output clipping and FP16 rounding of the backward rows."""
    W = [_h(np.asarray(weights, np.float64)[l], fp16) for l in range(LAYERS)]
    raw, acts = forward(weights, features, fp16)
    dw = np.array(dir_weight, np.float64)
    dw[:, 3] /= weight_scale
    loss, g = loss_and_grad(raw, dw)
    n = raw.shape[0]
    dz = np.zeros((n, DIM))
    dz[:, :OUTPUTS] = np.clip(g, -GRAD_CLIP, GRAD_CLIP)
    dz = _h(dz, fp16)
    grad = np.zeros((LAYERS, DIM, DIM))
    for l in range(LAYERS - 1, -1, -1):
        grad[l] = dz.T @ acts[l]
        if l > 0:
            dh = dz @ W[l]
            dz = _h(np.where(acts[l] > 0, dh, 0.0), fp16)
    return grad / n, loss.mean()


def adam(w, m, v, g, step, lr, b1=0.9, b2=0.99, eps=1e-8):
    """One Adam step (step counts from 1); returns new (w, m, v)."""
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    w = w - lr * (m / (1 - b1 ** step)) / (np.sqrt(v / (1 - b2 ** step)) + eps)
    return w, m, v
