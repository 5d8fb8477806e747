"""Problem ingestion on the GPU: QUBO::to_ising (qubo.cpp:33-69) formed by device
kernels straight into the model's device copy, and the dense derived arrays
(float32 mirror, +-1 bit rows) built on the device from the uploaded couplings."""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200.instances import geometric_betas

pytestmark = pytest.mark.gpu


def _qubo(n, seed, kind):
    rng = np.random.default_rng(seed)
    if kind == "pm1":  # symmetric +-2 off the diagonal: J = W/2 = +-1, the +-1 kernels
        U = np.triu(rng.choice([-2.0, 2.0], size=(n, n)), 1)
        return U + U.T + np.diag(rng.choice([-1.0, 0.0, 3.0], size=n))
    if kind == "asym":  # Q and Q^T differ, real entries spanning magnitudes
        return rng.normal(size=(n, n)) * np.exp(rng.uniform(-8, 8, size=(n, n)))
    return rng.integers(-3, 4, size=(n, n)).astype(np.float64)


@pytest.mark.parametrize("n", [1, 5, 33, 100, 257])
@pytest.mark.parametrize("kind", ["pm1", "asym", "int"])
def test_qubo_to_ising_on_device_equals_host(n, kind):
    Q = _qubo(n, 7 * n + len(kind), kind)
    host = qa.QUBO(Q).to_ising()
    dev = qa.QUBO(Q).to_ising_device()
    np.testing.assert_array_equal(dev.fields(), host.fields())
    assert dev.constant() == host.constant()
    np.testing.assert_array_equal(dev.couplings(), host.couplings())
    # the device copies drive identical anneals (J64 for energies, J32 / bit rows for sweeps)
    betas = geometric_betas(0.1, 3.0, 12)
    a = qa.Annealer(host, qa.AnnealSchedule.from_betas(betas)).run_reads(2, reads=3, seed=5)
    b = qa.Annealer(dev, qa.AnnealSchedule.from_betas(betas)).run_reads(2, reads=3, seed=5)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x.best_state.as_array(), y.best_state.as_array())
        assert x.best_energy == y.best_energy
        np.testing.assert_array_equal(np.asarray(x.energy_trace), np.asarray(y.energy_trace))
    if n >= 5:
        sched = qa.SQASchedule.from_vectors([2.0] * 8, np.linspace(2.0, 0.1, 8))
        s1 = qa.SQAAnnealer(host, sched, 8, 1).run_reads(1, 1, reads=2, seed=9)
        s2 = qa.SQAAnnealer(dev, sched, 8, 1).run_reads(1, 1, reads=2, seed=9)
        for x, y in zip(s1, s2):
            np.testing.assert_array_equal(x.best_state.as_array(), y.best_state.as_array())
            assert x.best_energy == y.best_energy
            np.testing.assert_array_equal(np.asarray(x.energy_trace), np.asarray(y.energy_trace))


def test_device_built_model_matches_oracle(oracle):
    """The device-converted +-1 model on the bit-row kernel equals the oracle's
    run on the host-converted model."""
    from test_gpu_parity_sa_sqa import oracle_model
    Q = _qubo(96, 3, "pm1")
    host = qa.QUBO(Q).to_ising()
    dev = qa.QUBO(Q).to_ising_device()
    om = oracle_model(oracle, host)
    steps, P = 12, 8
    betas = np.full(steps, 1.0 * P / 4.0)
    gammas = np.linspace(3.0, 0.05, steps)
    res = qa.SQAAnnealer(dev, qa.SQASchedule.from_vectors(betas, gammas), P, 1).run_reads(1, 1, reads=2, seed=31)
    for r in range(2):
        best, E, trace, _ = oracle.sqa_run(om, betas, gammas, P, 1, 1, 1, 31, r)
        np.testing.assert_array_equal(res[r].best_state.as_array(), best)
        assert res[r].best_energy == E
        np.testing.assert_array_equal(np.asarray(res[r].energy_trace), trace)


def test_solve_converts_qubo_on_device():
    rng = np.random.default_rng(4)
    Q = rng.normal(size=(40, 40))
    r = qa.solve(Q, method="sa", reads=3, seed=2, return_bits=True)
    ref = qa.solve(qa.QUBO(Q).to_ising(), method="sa", reads=3, seed=2)
    assert r.energies == ref.energies
    for a, b in zip(r.samples, ref.samples):
        np.testing.assert_array_equal(a, (b + 1) // 2)
    x = r.best_sample.astype(float)
    assert r.best_energy == pytest.approx(x @ Q @ x, abs=1e-9)
