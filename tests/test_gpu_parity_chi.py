"""SQA-Chi on the GPU against the CPU restatement, bit for bit: the pilot
chi_B scan (all probes batched), the schedule, the production anneal; and the
reference's own checks (tests/test_sqa_chi_annealer.cpp) through the GPU path."""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from test_gpu_parity_sa_sqa import make, oracle_model
from test_oracle_chi import ferro_chain, xorshift_sk

pytestmark = pytest.mark.gpu

CHI_CASES = [
    # kind, n, P, K, steps, spb, points, sweeps, burn
    ("dense", 64, 8, 2, 30, 3, 8, 10, 4),
    ("dense", 40, 5, 1, 20, 2, 6, 8, 2),
    ("dense_int", 48, 6, 2, 16, 2, 5, 6, 3),
    ("sparse", 96, 8, 2, 20, 2, 6, 8, 3),
    ("hubo", 36, 4, 1, 12, 2, 4, 6, 2),
]


def _compare(res, o):
    np.testing.assert_array_equal(np.asarray(res.scan_chi_B), o["scan_chi"])
    np.testing.assert_array_equal(np.asarray(res.scan_s), o["scan_s"])
    np.testing.assert_array_equal(np.asarray(res.scan_gamma), o["scan_gamma"])
    np.testing.assert_array_equal(np.asarray(res.beta_schedule), o["beta"])
    np.testing.assert_array_equal(np.asarray(res.gamma_schedule), o["gamma"])
    np.testing.assert_array_equal(np.asarray(res.s_schedule), o["s"])
    np.testing.assert_array_equal([res.s_star, res.gamma_star, res.j_perp_star, res.chi_floor, res.driver_A0],
                                  o["scalars"])
    np.testing.assert_array_equal(np.asarray(res.energy_trace), o["trace"])
    np.testing.assert_array_equal(res.best_state.as_array(), o["best"])
    assert res.best_energy == o["best_energy"]


@pytest.mark.parametrize("kind,n,P,K,steps,spb,points,sweeps,burn", CHI_CASES)
def test_chi_bit_exact(oracle, kind, n, P, K, steps, spb, points, sweeps, burn):
    model = make(kind, n, 41)
    om = oracle_model(oracle, model)
    beta, g0, g1, reads, seed = 0.4 * P, 3.0, 0.05, 2, 1357
    ann = qa.SQAChiAnnealer(model, P, K)
    res = ann.run_chi_reads(beta, g0, g1, steps, spb, points, sweeps, burn, reads=reads, seed=seed)
    for r in range(reads):
        _compare(res[r], oracle.chi_run(om, P, K, beta, g0, g1, steps, spb, points, sweeps, burn, seed, r))
    # a supplied chi_B curve replaces the pilot (the learned-schedule path)
    curve = np.linspace(1.0, 5.0, points) ** 2
    res2 = ann.run_chi_reads(beta, g0, g1, steps, spb, points, sweeps, burn, reads=reads, seed=seed, scan_chi=curve)
    for r in range(reads):
        _compare(res2[r], oracle.chi_run(om, P, K, beta, g0, g1, steps, spb, points, sweeps, burn, seed, r,
                                         scan_chi_in=curve))


def test_chi_rotated_production_bit_exact(oracle):
    """More rings than SMs and >= 200 production sweeps: the production anneal
    runs as rotated launches of ring groups; every read equals the oracle's."""
    model = make("dense", 40, 43)
    om = oracle_model(oracle, model)
    P, K, steps, spb, points, sweeps, burn = 4, 2, 30, 8, 5, 6, 2
    beta, g0, g1, reads, seed = 0.4 * P, 3.0, 0.05, 80, 2468
    ann = qa.SQAChiAnnealer(model, P, K)
    res = ann.run_chi_reads(beta, g0, g1, steps, spb, points, sweeps, burn, reads=reads, seed=seed)
    assert ann.last_stats.sweep_launches > 10  # ring groups, not one whole-grid launch (plus the pilot)
    for r in range(reads):
        _compare(res[r], oracle.chi_run(om, P, K, beta, g0, g1, steps, spb, points, sweeps, burn, seed, r))


def test_reference_chi_checks_on_gpu():
    # (A) schedule structure on the xorshift SK instance
    h, J = xorshift_sk(10)
    ann = qa.SQAChiAnnealer(qa.DenseIsing(h, J), 8, 4)
    ann.set_seed(2026)
    res = ann.run_chi(4.0, 4.0, 0.05, 120, 8, 12, 24, 8)
    assert len(res.scan_chi_B) == 12 and len(res.gamma_schedule) == 120 and len(res.energy_trace) == 120
    assert min(res.scan_chi_B) >= 0.0 and max(res.scan_chi_B) > min(res.scan_chi_B)
    assert res.scan_s[0] <= res.s_star <= res.scan_s[-1] and res.chi_floor > 0.0 and res.driver_A0 == 4.0
    g = np.asarray(res.gamma_schedule)
    assert np.all(np.diff(g) <= 1e-12) and abs(g[0] - 4.0) < 1e-9 and abs(g[-1] - 0.05) < 1e-6
    # (B), (C) exact ground states
    h, J = ferro_chain(12)
    a = qa.SQAChiAnnealer(qa.DenseIsing(h, J), 8, 4)
    a.set_seed(7)
    assert a.run_chi(4.0, 3.0, 0.05, 100, 10, 10, 20, 6).best_energy == -11.0
    ring = qa.SparseIsing(np.zeros(12), [(i, (i + 1) % 12, -1.0) for i in range(12)], 12)
    a = qa.SQAChiAnnealer(ring, 8, 4)
    a.set_seed(11)
    assert a.run_chi(4.0, 3.0, 0.05, 100, 10, 10, 20, 6).best_energy == -12.0
    # (D) degenerate range
    h, J = ferro_chain(6)
    a = qa.SQAChiAnnealer(qa.DenseIsing(h, J), 4, 2)
    a.set_seed(3)
    res = a.run_chi(0.5, 0.2, 0.15, 20, 4, 4, 4, 2)
    assert len(res.gamma_schedule) == 20 and all(np.isfinite(res.gamma_schedule)) and min(res.gamma_schedule) > 0


def test_chi_argument_errors():
    h, J = ferro_chain(6)
    a = qa.SQAChiAnnealer(qa.DenseIsing(h, J), 4, 1)
    with pytest.raises(ValueError, match="num_steps"):
        a.run_chi(1.0, 2.0, 0.1, 1)
    with pytest.raises(ValueError, match="gamma_start > gamma_end"):
        a.run_chi(1.0, 0.1, 2.0)
    with pytest.raises(ValueError, match="scan_points"):
        a.run_chi(1.0, 2.0, 0.1, 10, 2, 3)
