"""Seeded synthetic problem instances (benchmark and test workloads).

The shapes and value distributions follow the benchmark configurations of the
sweep engine: dense Sherrington-Kirkpatrick (J in {-1,+1}), random 3-regular
sparse graphs, random 3-body + 2-body HUBO.  No public data set is involved.
"""
from __future__ import annotations

import numpy as np


def sk_dense(n: int, seed: int, h_sigma: float = 0.0, h_float32: bool = True):
    rng = np.random.default_rng(seed)
    J = rng.choice([-1.0, 1.0], size=(n, n))
    J = np.triu(J, 1)
    J = J + J.T
    h = rng.normal(0.0, h_sigma, n) if h_sigma > 0 else np.zeros(n)
    if h_float32:
        h = h.astype(np.float32).astype(np.float64)
    return h, J


def dense_real(n: int, seed: int):
    rng = np.random.default_rng(seed)
    J = rng.uniform(-1.0, 1.0, size=(n, n))
    J = np.triu(J, 1)
    J = J + J.T
    h = rng.normal(0.0, 0.3, n)
    return h, J


def regular3(n: int, seed: int, h_choices=(-0.5, 0.0, 0.5)):
    """Random 3-regular graph (configuration model with rejection), J in {-1,+1}."""
    rng = np.random.default_rng(seed)
    assert n % 2 == 0
    while True:
        stubs = np.repeat(np.arange(n), 3)
        rng.shuffle(stubs)
        pairs = stubs.reshape(-1, 2)
        if np.any(pairs[:, 0] == pairs[:, 1]):
            continue
        a = np.minimum(pairs[:, 0], pairs[:, 1])
        b = np.maximum(pairs[:, 0], pairs[:, 1])
        key = a * n + b
        if len(np.unique(key)) != len(key):
            continue
        break
    w = rng.choice([-1.0, 1.0], size=len(a))
    h = rng.choice(np.asarray(h_choices, dtype=np.float64), size=n)
    edges = [(int(x), int(y), float(v)) for x, y, v in zip(a, b, w)]
    return h, edges


def hubo_random(n: int, seed: int, integer: bool = False):
    """3n distinct 3-body terms (J in {-1,+1}) + 2n 2-body terms (J ~ U(-1,1),
    or {-1,+1} when integer) + h ~ N(0, 0.2^2) (or {-1,0,1})."""
    rng = np.random.default_rng(seed)
    terms = {}
    while len([k for k in terms if len(k) == 3]) < 3 * n:
        t = tuple(sorted(rng.choice(n, size=3, replace=False).tolist()))
        if t not in terms:
            terms[t] = float(rng.choice([-1.0, 1.0]))
    cnt2 = 0
    while cnt2 < 2 * n:
        t = tuple(sorted(rng.choice(n, size=2, replace=False).tolist()))
        if t in terms:
            continue
        terms[t] = float(rng.choice([-1.0, 1.0])) if integer else float(rng.uniform(-1.0, 1.0))
        cnt2 += 1
    if integer:
        h = rng.choice([-1.0, 0.0, 1.0], size=n)
    else:
        h = rng.normal(0.0, 0.2, n)
    for i in range(n):
        if h[i] != 0.0:
            terms[(i,)] = float(h[i])
    return terms


def geometric_betas(b0: float, b1: float, steps: int):
    k = np.arange(steps)
    return b0 * (b1 / b0) ** (k / max(steps - 1, 1))
