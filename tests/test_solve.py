"""solve() and its schedule helpers (python/qanneal/solver.py semantics)."""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200 import solver
from qlatanneal_b200.instances import regular3, sk_dense


def test_schedule_helpers():
    s = qa.auto_schedule_sqa(10, 0.1, 4.0, 5.0, 0.01)
    np.testing.assert_allclose(s.betas, np.linspace(0.1, 4.0, 10))
    np.testing.assert_allclose(s.gammas, np.geomspace(5.0, 0.01, 10))
    a = qa.auto_schedule_sa(5, 0.5, 2.5)
    np.testing.assert_allclose(a.betas, [0.5, 1.0, 1.5, 2.0, 2.5])
    assert qa.j_perp_from_beta_gamma(16.0, 3.0, 32) == pytest.approx(0.5 * np.log(1.0 / np.tanh(1.5)))
    h, J = sk_dense(20, 1)
    d = qa.DenseIsing(h, J)
    lad = qa.auto_ladder_sqa_tuned(d, replicas=6)
    assert len(lad.betas) == 6 and np.all(np.diff(lad.betas) > 0) and np.all(np.diff(lad.gammas) < 0)
    b, jp0, jp1 = qa.optimal_j_perp_params(d, trotter_slices=16)
    assert b == max(4.0 / qa.j_rms_from_problem(d), 1.0) and jp1 > jp0 > 0
    assert qa.j_rms_from_problem(d) == pytest.approx(1.0)
    with pytest.raises(ValueError):
        solver._mode_params("slow")


def test_normalize_problem_forms():
    Q = np.array([[1.0, -2.0], [0.0, 3.0]])
    for prob in (Q, qa.QUBO(Q), {(0, 0): 1.0, (0, 1): -2.0, (1, 1): 3.0}, [(0, 0, 1.0), (0, 1, -2.0), (1, 1, 3.0)]):
        ising, order, bits = solver._normalize_problem(prob)
        assert bits and order == [0, 1]
        x = np.array([1, 0])
        s = 2 * x - 1
        assert ising.energy(s) == pytest.approx(x @ Q @ x)
    hubo, order, bits = solver._normalize_problem({(0, 1, 2): 1.0, 3: 0.5})
    assert isinstance(hubo, qa.HigherOrderIsing) and not bits and order == [0, 1, 2, 3]
    with pytest.raises(ValueError):
        solver._normalize_problem("nope")
    with pytest.raises(ValueError):
        qa.solve(qa.DenseIsing(np.zeros(2), np.zeros((2, 2))), return_bits=True)
    with pytest.raises(NotImplementedError):
        qa.solve(Q, method="ctpimc")


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["sa", "sqa", "sqapt", "sqa_chi"])
def test_solve_methods_on_gpu(method):
    h, J = sk_dense(40, 3)
    d = qa.DenseIsing(h, J)
    kw = dict(trotter_slices=8, sweeps_per_beta=2, worldline_sweeps=1, pt_steps=10, chi_scan_points=6,
              chi_scan_sweeps=6, chi_scan_burn=2, optimal_num_steps=30, replicas=3 if method == "sqapt" else 1)
    r = qa.solve(d, method=method, reads=5, seed=77, **kw)
    assert r.method == method and len(r.samples) == 5 and len(r.energies) == 5
    assert r.best_energy == min(r.energies)
    assert r.best_energy == pytest.approx(d.energy(r.best_sample), abs=1e-9)
    assert r.trace is not None and len(r.trace) > 0
    # read r of a batched solve == a single-read solve seeded seed + r (solver.py:679-681)
    one = qa.solve(d, method=method, reads=1, seed=79, **kw)
    assert one.energies[0] == r.energies[2]
    np.testing.assert_array_equal(one.samples[0], r.samples[2])


@pytest.mark.gpu
def test_solve_qubo_bits_and_sparse():
    rng = np.random.default_rng(0)
    Q = rng.normal(size=(12, 12))
    r = qa.solve(Q, method="sa", reads=3, seed=1, return_bits=True)
    assert set(np.unique(r.best_sample)) <= {0, 1}
    x = r.best_sample.astype(float)
    assert r.best_energy == pytest.approx(x @ Q @ x, abs=1e-9)
    h, e = regular3(64, 2)
    s = qa.SparseIsing(h, e, 64)
    r = qa.solve(s, method="sqa", reads=4, seed=3, trotter_slices=8, sweeps_per_beta=2, worldline_sweeps=1)
    assert r.best_energy == pytest.approx(s.energy(r.best_sample), abs=1e-9)
