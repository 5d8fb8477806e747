"""Statistics for comparing sampled energies (test infrastructure).

* ``two_sample_chi2``: two samples of a discrete energy variable, levels pooled
  into bins with at least 10 observations in the pair (tail bins merged), the
  chi-square test of homogeneity; returns (p-value, bins).
* ``wilson``: the 95% Wilson interval of a binomial proportion.
* ``ising_levels`` / ``trotter_mean_energy_levels``: exact enumeration of the
  Boltzmann distribution of a small Ising model and of the mean slice energy
  under the Trotterized action of a small ring (n * P <= 20).
* ``gof_chi2``: one sample against exact level probabilities.
"""
from __future__ import annotations

import math

import numpy as np
from scipy.stats import chi2, chi2_contingency


def wilson(k: int, n: int, z: float = 1.96):
    p = k / n
    d = 1.0 + z * z / n
    c = (p + z * z / (2 * n)) / d
    w = z * math.sqrt(p * (1 - p) / n + z * z / (4 * n * n)) / d
    return c - w, c + w


def mean_ci(x, z: float = 1.96):
    x = np.asarray(x, float)
    return x.mean(), z * x.std(ddof=1) / math.sqrt(len(x))


def two_sample_chi2(a, b, decimals: int = 9):
    a, b = np.round(np.asarray(a, float), decimals), np.round(np.asarray(b, float), decimals)
    levels = np.unique(np.concatenate([a, b]))
    ca = np.array([(a == v).sum() for v in levels], float)
    cb = np.array([(b == v).sum() for v in levels], float)
    bins, acc = [], np.zeros(2)
    for x, y in zip(ca, cb):
        acc += (x, y)
        if acc.sum() >= 10 and acc.min() >= 1:
            bins.append(acc.copy())
            acc[:] = 0
    if acc.sum():
        if bins:
            bins[-1] += acc
        else:
            bins.append(acc.copy())
    tab = np.array(bins).T
    if tab.shape[1] < 2:
        return 1.0, tab.shape[1]
    return float(chi2_contingency(tab)[1]), tab.shape[1]


def all_states(n: int) -> np.ndarray:
    return 1 - 2 * ((np.arange(2 ** n)[:, None] >> np.arange(n)) & 1)


def ising_energies(h, J, c=0.0) -> np.ndarray:
    s = all_states(len(h))
    return c + s @ np.asarray(h, float) + 0.5 * np.einsum("ki,ij,kj->k", s, np.asarray(J, float), s)


def ising_levels(h, J, beta: float, decimals: int = 9) -> dict:
    """{E: probability} of exp(-beta E) over all 2^n states."""
    E = ising_energies(h, J)
    w = np.exp(-beta * (E - E.min()))
    w /= w.sum()
    out: dict = {}
    for e, p in zip(np.round(E, decimals), w):
        out[e] = out.get(e, 0.0) + p
    return out


def trotter_mean_energy_levels(h, J, beta: float, gamma: float, P: int, decimals: int = 9) -> dict:
    """{(1/P) sum_t E(s_t): probability} under the Trotterized action
    S = (beta/P) sum_t E(s_t) - J_perp sum_t sum_i s_t,i s_t+1,i (periodic in t),
    J_perp = 1/2 ln coth(beta Gamma / P) (sqa_annealer.cpp:66-70), by direct
    enumeration of all 2^(nP) ring states (n P <= 20)."""
    n = len(h)
    assert n * P <= 20
    E = ising_energies(h, J)                      # slice energy by slice state index
    S = all_states(n)
    overlap = S @ S.T                             # sum_i s_i s'_i by pair of slice states
    jp = 0.5 * math.log(1.0 / math.tanh(max(beta * gamma / P, 1e-12)))
    ring = np.arange(2 ** (n * P), dtype=np.int64)
    mask = (1 << n) - 1
    sl = [(ring >> (n * t)) & mask for t in range(P)]
    esum = sum(E[x] for x in sl)
    bond = sum(overlap[sl[t], sl[(t + 1) % P]] for t in range(P))
    logw = -(beta / P) * esum + jp * bond
    w = np.exp(logw - logw.max())
    w /= w.sum()
    out: dict = {}
    for e, p in zip(np.round(esum / P, decimals), w):
        out[e] = out.get(e, 0.0) + p
    return out


def gof_chi2(samples, levels: dict, decimals: int = 9):
    """Chi-square p-value of samples against level probabilities, tail levels
    merged until each expected count is >= 5; returns (p, bins)."""
    keys = sorted(levels)
    exp_c = np.array([levels[k] for k in keys]) * len(samples)
    pos = {k: i for i, k in enumerate(keys)}
    obs = np.zeros(len(keys))
    for e in np.round(np.asarray(samples, float), decimals):
        obs[pos[e]] += 1
    bo, be, co, ce = [], [], 0.0, 0.0
    for o, e in zip(obs, exp_c):
        co += o
        ce += e
        if ce >= 5.0:
            bo.append(co)
            be.append(ce)
            co = ce = 0.0
    if ce > 0:
        bo[-1] += co
        be[-1] += ce
    bo, be = np.array(bo), np.array(be)
    stat = float(np.sum((bo - be) ** 2 / be))
    return float(chi2.sf(stat, len(bo) - 1)), len(bo)
