"""The initial local fields on the tensor cores (tc_fields_kernel: tcgen05
int8 MMAs, int32 accumulators in TMEM) against the float64 field init.

DenseIsing::compute_local_fields (dense_ising.cpp:64-83) of every Trotter
cell of a run.  For integer couplings in [-127, 127] the int8 product is
exact, so runs of the generic ring kernels (dense integer couplings, cluster
sweeps, SQA-PT, the SQA-Chi pilot with its fresh ring per scan point) must be
bit for bit the runs with the tensor-core path switched off
(QA_DISABLE_TC_INIT), and the oracle's.
"""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200.instances import sk_dense
from test_gpu_parity_sa_sqa import oracle_model

pytestmark = pytest.mark.gpu


def _int_dense(n, seed, scale=(-3.0, -1.0, 1.0, 2.0, 5.0)):
    rng = np.random.default_rng(seed)
    J = np.triu(rng.choice(scale, size=(n, n)), 1)
    return qa.DenseIsing(rng.choice([-1.0, 0.0, 1.0], size=n), J + J.T, 0.5)


def _sqa(model, P, K, cls, reads, seed):
    betas, gammas = np.full(6, 0.3 * P), np.linspace(2.0, 0.2, 6)
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(betas, gammas), P, K)
    return ann.run_reads(1, 1, cluster_sweeps=cls, reads=reads, seed=seed), betas, gammas


@pytest.mark.parametrize("n,P,K,cls", [(70, 6, 1, 0), (300, 8, 2, 0), (129, 3, 1, 1), (600, 4, 1, 0)])
def test_tc_init_equals_float64_init(oracle, monkeypatch, n, P, K, cls):
    model = _int_dense(n, 7 + n)
    res, betas, gammas = _sqa(model, P, K, cls, 5, 33)
    with monkeypatch.context() as mp:
        mp.setenv("QA_DISABLE_TC_INIT", "1")
        ref, _, _ = _sqa(model, P, K, cls, 5, 33)
    for a, b in zip(res, ref):
        np.testing.assert_array_equal(a.best_state.as_array(), b.best_state.as_array())
        assert a.best_energy == b.best_energy
        np.testing.assert_array_equal(np.asarray(a.energy_trace), np.asarray(b.energy_trace))
    om = oracle_model(oracle, model)
    best, E, trace, _ = oracle.sqa_run(om, betas, gammas, P, K, 1, 1, 33, 0, cls=cls)
    np.testing.assert_array_equal(res[0].best_state.as_array(), best)
    np.testing.assert_array_equal(np.asarray(res[0].energy_trace), trace)


def test_tc_init_instance_set_and_pt(monkeypatch):
    """Several problems of uneven size in one launch (one tensor-core launch
    per problem over its rings) and SQA-PT."""
    models = [_int_dense(n, n) for n in (40, 257, 130)]
    sched = qa.SQASchedule.from_vectors(np.full(5, 2.0), np.linspace(2.0, 0.1, 5))

    def run():
        a = qa.BatchRunner().sqa(models, sched, 4, 1, 1, 1, cluster_sweeps=1, reads=3, seed=8)
        b = qa.SQAParallelTemperingAnnealer(models[1], [0.5, 1.0, 2.0], [2.0, 1.0, 0.2], 4).run_reads(
            1, 1, 6, 2, cluster_sweeps=1, reads=2, seed=9)
        return a, b

    a1, b1 = run()
    with monkeypatch.context() as mp:
        mp.setenv("QA_DISABLE_TC_INIT", "1")
        a2, b2 = run()
    for x, y in zip(a1, a2):
        for r, s in zip(x, y):
            assert r.best_energy == s.best_energy and r.energy_trace == s.energy_trace
    for r, s in zip(b1, b2):
        assert r.best_energy == s.best_energy and list(r.final_energies) == list(s.final_energies)


def test_tc_init_chi_pilot_equals_float64_init(monkeypatch):
    """The SQA-Chi pilot starts a fresh ring at every scan point; at n = 1600,
    P = 64 (too large for the bit-packed kernel) its fields come from the
    tensor cores.  The chi_B curves must not change."""
    from qlatanneal_b200 import learned
    h, J = sk_dense(1600, 77)
    m = qa.DenseIsing(h, J)
    kw = dict(points=6, sweeps=4, burn=2, reads=2, seed=5)
    c1 = learned.pilot_curves([m], 4.0, 3.0, 0.1, 64, **kw)
    with monkeypatch.context() as mp:
        mp.setenv("QA_DISABLE_TC_INIT", "1")
        c2 = learned.pilot_curves([m], 4.0, 3.0, 0.1, 64, **kw)
    np.testing.assert_array_equal(c1, c2)
