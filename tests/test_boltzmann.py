"""Sampled distributions against exact enumeration (n = 10).

At Gamma -> 0 the Trotter slices of a ring lock together (J_perp -> infinity)
and a worldline move is a classical Metropolis flip with
Delta S = beta Delta E, so the final state of each SQA-PT rung samples the
classical Boltzmann distribution exp(-beta_r E) (swaps between rungs keep it:
with aligned rings the bond terms cancel).  The energies of many independent
reads are binned by energy level and compared with the enumerated
probabilities by a chi-square test; the oracle on the CPU and the CUDA engine
are each checked.
"""
import math

import numpy as np
import pytest

from qlatanneal_b200.instances import sk_dense

N, P, STEPS, READS = 10, 2, 300, 4000
BETAS = [0.25, 0.5]
GAMMAS = [1e-6, 1e-6]


def _instance():
    h, J = sk_dense(N, 404)
    rng = np.random.default_rng(405)
    h = rng.choice([-1.0, 0.0, 1.0], size=N)
    return h, J


def _levels(h, J, beta):
    """Exact energy-level probabilities {E: p} of exp(-beta E) over all 2^n states."""
    s = 1 - 2 * ((np.arange(2 ** N)[:, None] >> np.arange(N)) & 1)
    E = s @ h + 0.5 * np.einsum("ki,ij,kj->k", s, J, s)
    w = np.exp(-beta * (E - E.min()))
    w /= w.sum()
    out = {}
    for e, p in zip(np.round(E, 9), w):
        out[e] = out.get(e, 0.0) + p
    return out


def _chi2_pvalue(samples, levels):
    """Chi-square p-value of sampled energies against level probabilities,
    tail levels merged until every expected count is >= 5."""
    from scipy.stats import chi2
    keys = sorted(levels)
    exp_c = np.array([levels[k] for k in keys]) * len(samples)
    idx = {k: i for i, k in enumerate(keys)}
    obs = np.zeros(len(keys))
    for e in np.round(samples, 9):
        obs[idx[e]] += 1
    bins_o, bins_e, co, ce = [], [], 0.0, 0.0
    for o, e in zip(obs, exp_c):
        co += o
        ce += e
        if ce >= 5.0:
            bins_o.append(co)
            bins_e.append(ce)
            co = ce = 0.0
    if ce > 0:
        bins_o[-1] += co
        bins_e[-1] += ce
    bins_o, bins_e = np.array(bins_o), np.array(bins_e)
    stat = float(np.sum((bins_o - bins_e) ** 2 / bins_e))
    return float(chi2.sf(stat, len(bins_o) - 1)), len(bins_o)


def _check(final_E):
    h, J = _instance()
    for k, beta in enumerate(BETAS):
        p, dof = _chi2_pvalue(final_E[:, k], _levels(h, J, beta))
        assert dof >= 5
        assert p > 1e-4, (beta, p)
        # the mean energy as well, within 5 standard errors
        lv = _levels(h, J, beta)
        mu = sum(e * q for e, q in lv.items())
        sd = math.sqrt(sum((e - mu) ** 2 * q for e, q in lv.items()))
        assert abs(final_E[:, k].mean() - mu) < 5 * sd / math.sqrt(len(final_E))


def test_oracle_samples_boltzmann(oracle):
    h, J = _instance()
    om = oracle.dense(h, J)
    fE = np.array([oracle.sqapt_run(om, BETAS, GAMMAS, P, 1, 1, STEPS, 1, 77, r)[2] for r in range(READS)])
    _check(fE)


@pytest.mark.gpu
def test_gpu_samples_boltzmann():
    import qlatanneal_b200 as qa
    h, J = _instance()
    ann = qa.SQAParallelTemperingAnnealer(qa.DenseIsing(h, J), BETAS, GAMMAS, P)
    res = ann.run_reads(1, 1, STEPS, 1, reads=READS, seed=77)
    _check(np.array([r.final_energies for r in res]))
