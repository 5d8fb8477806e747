"""Edge sizes on the GPU against the oracle: one and two spins, ragged sizes
around the 32-spin blocks, a single Trotter slice, and large sparse / HUBO /
dense instances (the kernels' global-memory and bits-from-L2 forms)."""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200.instances import geometric_betas, hubo_random, regular3, sk_dense
from test_gpu_parity_sa_sqa import oracle_model

pytestmark = pytest.mark.gpu


def _tiny(kind, n, seed):
    rng = np.random.default_rng(seed)
    h = rng.choice([-0.5, 0.0, 0.5], size=n)
    if kind == "dense":
        J = np.triu(rng.choice([-1.0, 1.0], size=(n, n)), 1)
        return qa.DenseIsing(h, J + J.T, 0.25)
    if kind == "sparse":
        e = [(i, (i + 1) % n, float(rng.choice([-1.0, 1.0]))) for i in range(n - 1)]
        return qa.SparseIsing(h, e, n, -1.0)
    terms = {(i,): float(h[i]) for i in range(n)}
    if n >= 2:
        terms[(0, n - 1)] = 0.75
    if n >= 3:
        terms[(0, 1, n - 1)] = -1.0
    return qa.HigherOrderIsing(terms, n)


@pytest.mark.parametrize("kind", ["dense", "sparse", "hubo"])
@pytest.mark.parametrize("n", [1, 2, 3, 31, 33])
def test_tiny_models_match_oracle(oracle, kind, n):
    model = _tiny(kind, n, 5 * n + len(kind))
    om = oracle_model(oracle, model)
    betas = geometric_betas(0.2, 3.0, 6)
    sa = qa.Annealer(model, qa.AnnealSchedule.from_betas(betas)).run_reads(2, reads=2, seed=3)
    for r in range(2):
        best, E, trace, _ = oracle.sa_run(om, betas, 2, 3, r)
        np.testing.assert_array_equal(sa[r].best_state.as_array(), best)
        np.testing.assert_array_equal(np.asarray(sa[r].energy_trace), trace)
    for P, K in ((1, 1), (3, 2)):
        sb, sg = np.full(5, 1.5 * P), np.linspace(2.0, 0.2, 5)
        res = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(sb, sg), P, K).run_reads(1, 1, reads=2, seed=7)
        for r in range(2):
            best, E, trace, _ = oracle.sqa_run(om, sb, sg, P, K, 1, 1, 7, r)
            np.testing.assert_array_equal(res[r].best_state.as_array(), best)
            np.testing.assert_array_equal(np.asarray(res[r].energy_trace), trace)
    pb, pg = np.array([0.5, 2.0]), np.array([1.5, 0.4])
    pt = qa.SQAParallelTemperingAnnealer(model, pb, pg, 2).run_reads(1, 1, 4, 1, reads=1, seed=9)
    best, E, fE, fs, avg, swp, _ = oracle.sqapt_run(om, pb, pg, 2, 1, 1, 4, 1, 9, 0)
    np.testing.assert_array_equal(pt[0].best_state.as_array(), best)
    np.testing.assert_array_equal(np.asarray(pt[0].average_energy_trace), avg)
    np.testing.assert_array_equal(np.asarray(pt[0].swap_acceptance_trace), swp)


def test_large_sparse_and_hubo_match_oracle(oracle):
    """n = 20000 sparse (more spins than the shared-memory forms hold) and an
    n = 6000 HUBO: a few steps, read 0, against the oracle."""
    h, e = regular3(20000, 4)
    sp = qa.SparseIsing(h, e, 20000)
    hu = qa.HigherOrderIsing(hubo_random(6000, 5), 6000)
    for model in (sp, hu):
        om = oracle_model(oracle, model)
        sb, sg = np.full(3, 2.0), np.linspace(1.5, 0.5, 3)
        res = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(sb, sg), 4, 1).run_reads(1, 1, reads=1, seed=11)
        best, E, trace, _ = oracle.sqa_run(om, sb, sg, 4, 1, 1, 1, 11, 0)
        np.testing.assert_array_equal(res[0].best_state.as_array(), best)
        np.testing.assert_array_equal(np.asarray(res[0].energy_trace), trace)


def test_large_dense_matches_oracle(oracle):
    """Dense +-1 n = 4096 (couplings as bits from L2, int16 fields) and a
    real-valued dense n = 3000 (float fields in global memory)."""
    h, J = sk_dense(4096, 6)
    d1 = qa.DenseIsing(h, J)
    rng = np.random.default_rng(8)
    A = rng.normal(size=(3000, 3000))
    d2 = qa.DenseIsing(rng.normal(size=3000), np.triu(A, 1) + np.triu(A, 1).T)
    for model in (d1, d2):
        om = oracle_model(oracle, model)
        sb, sg = np.full(2, 1.0), np.array([1.0, 0.3])
        res = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(sb, sg), 4, 1).run_reads(1, 1, reads=1, seed=13)
        best, E, trace, _ = oracle.sqa_run(om, sb, sg, 4, 1, 1, 1, 13, 0)
        np.testing.assert_array_equal(res[0].best_state.as_array(), best)
        np.testing.assert_array_equal(np.asarray(res[0].energy_trace), trace)
