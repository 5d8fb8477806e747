"""Incremental local-field updates over a long random walk of flips
(test_higher_order_ising.cpp:149-167): the reference's float64 cache stays
within 1e-7 of a recompute; the engine's float32 cache (this restatement, bit
for bit the GPU's) stays within a float32-sized bound of the float64 recompute
of the same float32 couplings.  The GPU-side drift check reports the same
quantity after a run."""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200.instances import hubo_random, regular3


def _instance(kind, n, rng):
    h = rng.normal(0.0, 0.5, size=n)
    if kind == "hubo":
        terms = {}
        for _ in range(3 * n):
            vs = tuple(sorted(rng.choice(n, size=int(rng.integers(2, 5)), replace=False).tolist()))
            terms[vs] = float(rng.uniform(-1.0, 1.0))
        return h, [(k, v) for k, v in terms.items()] + [((i,), float(h[i])) for i in range(n)]
    if kind == "dense":
        A = rng.uniform(-1.0, 1.0, size=(n, n))
        return h, np.triu(A, 1) + np.triu(A, 1).T
    e = [(i, (i + 1) % n, float(rng.uniform(-1, 1))) for i in range(n)]
    e += [(i, (i + 3) % n, float(rng.uniform(-1, 1))) for i in range(0, n, 2)]
    return h, e


def _model(lib, kind, n, data):
    h, x = data
    if kind == "hubo":
        return lib.hubo(n, x)
    if kind == "dense":
        return lib.dense(h, x)
    return lib.sparse(n, h, x)


@pytest.mark.parametrize("kind", ["hubo", "dense", "sparse"])
def test_field_drift_over_2000_flips(oracle, ref, kind):
    rng = np.random.default_rng(0xC0FFEE)
    worst32 = 0.0
    for n in (5, 8, 12, 20):
        for _ in range(5):
            data = _instance(kind, n, rng)
            om, rm = _model(oracle, kind, n, data), _model(ref, kind, n, data)
            s = rng.choice(np.array([-1, 1], np.int8), size=n)
            g = oracle.fields(om, s)                      # float32 cache, the engine's
            s64 = s.copy()
            f64 = rm.fields(s64)                          # the reference's float64 cache
            for _ in range(2000):
                i = int(rng.integers(n))
                oracle.flip_update(om, s, g, i)
                old = int(s64[i])
                s64[i] = -s64[i]
                rm.update_fields(f64, s64, i, old)
            np.testing.assert_array_equal(s, s64)
            # the reference's own property: within 1e-7 of a float64 recompute
            assert np.max(np.abs(f64 - rm.fields(s64))) < 1e-7
            # float32 cache vs the float64 recompute of the same float32 couplings
            worst32 = max(worst32, float(np.max(np.abs(g.astype(np.float64) - oracle.fields(om, s)))))
    assert worst32 < 1e-4, worst32


@pytest.mark.gpu
def test_gpu_drift_check():
    h, e = regular3(256, 3)
    rng = np.random.default_rng(4)
    real = qa.SparseIsing(h, [(a, b, w * rng.uniform(0.3, 1.2)) for a, b, w in e], 256)
    hubo = qa.HigherOrderIsing(hubo_random(128, 7), 128)
    integer = qa.HigherOrderIsing(hubo_random(128, 7, integer=True), 128)
    sched = qa.SQASchedule.from_vectors(np.full(30, 3.0), np.linspace(2.0, 0.1, 30))
    betas = qa.AnnealSchedule.from_betas(np.linspace(0.2, 3.0, 30))
    try:
        qa.set_drift_check(1e-2)
        for m in (real, hubo):
            a = qa.SQAAnnealer(m, sched, 8, 1)
            a.run_reads(1, 1, reads=4, seed=1)
            assert 0.0 < a.last_stats.max_field_drift < 1e-3
            b = qa.Annealer(m, betas)
            b.run_reads(2, reads=4, seed=1)
            assert 0.0 < b.last_stats.max_field_drift < 1e-3
            c = qa.SQAParallelTemperingAnnealer(m, [0.5, 2.0], [1.5, 0.3], 4)
            c.run_reads(1, 1, 10, 2, reads=2, seed=1)
            assert 0.0 < c.last_stats.max_field_drift < 1e-3
        a = qa.SQAAnnealer(integer, sched, 8, 1)
        a.run_reads(1, 1, reads=4, seed=1)
        assert a.last_stats.max_field_drift == 0.0  # integer sums are exact in float32
        qa.set_drift_check(1e-12)
        with pytest.raises(qa.FieldDriftError):
            qa.SQAAnnealer(hubo, sched, 8, 1).run_reads(1, 1, reads=4, seed=1)
    finally:
        qa.set_drift_check(0.0)
    a = qa.SQAAnnealer(hubo, sched, 8, 1)
    a.run_reads(1, 1, reads=4, seed=1)
    assert a.last_stats.max_field_drift == 0.0
