"""TEST INFRASTRUCTURE ONLY: float64 restatement of the chi_B-curve MLP.

Forward pass, Gaussian negative log-likelihood and hand-written backprop in
numpy float64, used to check the gradients computed by the CUDA kernels
(qlatanneal_b200/csrc/qa_mlp.cuh).  The weights it multiplies are the
bfloat16-rounded ones the kernels read; the loss clamps the log-variance to
[-12, 12] with zero gradient outside, as the kernels do.  Its own backprop is
checked against central finite differences in the tests.
"""
from __future__ import annotations

import numpy as np


def bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(params: np.ndarray, dims):
    out, off = [], 0
    for l in range(len(dims) - 1):
        k, n = dims[l], dims[l + 1]
        W = params[off:off + k * n].reshape(k, n)
        off += k * n
        b = params[off:off + n]
        off += n
        out.append((W, b))
    return out


def forward(params: np.ndarray, dims, X: np.ndarray, bf16: bool = True):
    acts = [np.asarray(X, np.float64)]
    layers = unpack(np.asarray(params), dims)
    for l, (W, b) in enumerate(layers):
        Wq = (bf16_round(W.astype(np.float32)) if bf16 else W).astype(np.float64)
        z = acts[-1] @ Wq + b.astype(np.float64)
        acts.append(np.maximum(z, 0.0) if l + 1 < len(layers) else z)
    return acts


def loss_and_grads(params: np.ndarray, dims, X: np.ndarray, T: np.ndarray, bf16: bool = True):
    """Mean Gaussian NLL over [mu | s] outputs and d loss / d params (float64)."""
    acts = forward(params, dims, X, bf16)
    Y = acts[-1]
    B, M2 = Y.shape
    M = M2 // 2
    mu, sr = Y[:, :M], Y[:, M:]
    s = np.clip(sr, -12.0, 12.0)
    e = np.exp(-s)
    d = np.asarray(T, np.float64) - mu
    loss = float(np.mean(0.5 * (e * d * d + s)))
    inv = 1.0 / (B * M)
    dY = np.concatenate([-e * d * inv, np.where((sr > -12) & (sr < 12), 0.5 * (1.0 - e * d * d) * inv, 0.0)], 1)
    layers = unpack(np.asarray(params), dims)
    grads = []
    dz = dY
    for l in range(len(layers) - 1, -1, -1):
        W, _ = layers[l]
        Wq = (bf16_round(W.astype(np.float32)) if bf16 else W).astype(np.float64)
        gW = acts[l].T @ dz
        gb = dz.sum(0)
        grads.append((gW, gb))
        if l > 0:
            dz = (dz @ Wq.T) * (acts[l] > 0.0)
    flat = []
    for gW, gb in reversed(grads):
        flat.append(gW.reshape(-1))
        flat.append(gb)
    return loss, np.concatenate(flat)


def finite_difference(params: np.ndarray, dims, X, T, idx, eps=1e-6):
    """Central difference of the float64 (unrounded-weight) loss at params[idx]."""
    p = np.asarray(params, np.float64).copy()
    out = []
    for i in idx:
        old = p[i]
        p[i] = old + eps
        lp, _ = loss_and_grads(p, dims, X, T, bf16=False)
        p[i] = old - eps
        lm, _ = loss_and_grads(p, dims, X, T, bf16=False)
        p[i] = old
        out.append((lp - lm) / (2 * eps))
    return np.array(out)


def adam_step(params, grads, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update in float32 with bias corrections 1 - b^step (Kingma & Ba, 2015)."""
    f = np.float32
    p, g = np.asarray(params, f), np.asarray(grads, f)
    m = f(b1) * np.asarray(m, f) + f(1.0 - b1) * g
    v = f(b2) * np.asarray(v, f) + f(1.0 - b2) * g * g
    c1, c2 = f(1.0 - b1 ** step), f(1.0 - b2 ** step)
    p = p - f(lr) * (m / c1) / (np.sqrt(v / c2) + f(eps))
    return p.astype(f), m, v
