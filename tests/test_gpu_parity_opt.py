"""SQAAnnealer.run_optimal on the GPU against the CPU restatement, bit for bit
(sqa_annealer.cpp:499-952): beta ramp, budget calibration (eps_tilde <= 0) or
online J_perp updates (eps_tilde > 0), chi_B from the bond-sum samples."""
import os

import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200.instances import sk_dense
from test_gpu_parity_sa_sqa import REAL_KINDS, make, oracle_model

pytestmark = pytest.mark.gpu

OPT_CASES = [
    # kind, n, P, K, eps_tilde, sweeps/step, worldline, cluster, probes, calib sweeps, steps
    ("dense", 64, 8, 1, 0.0, 2, 1, 0, 8, 4, 30),
    ("dense", 96, 16, 2, 0.02, 1, 1, 0, 6, 3, 24),
    ("dense", 48, 32, 1, 0.0, 1, 0, 0, 5, 2, 20),
    ("dense_h", 70, 6, 1, 0.0, 1, 1, 1, 8, 4, 30),
    ("dense_int", 48, 12, 1, 0.05, 1, 0, 2, 4, 2, 16),
    ("dense_hwide", 40, 4, 1, 0.0, 1, 1, 0, 6, 3, 20),
    ("sparse", 128, 8, 1, 0.0, 1, 1, 0, 8, 4, 30),
    ("sparse", 96, 16, 2, 0.03, 1, 0, 0, 4, 2, 18),
    ("sparse_real", 96, 6, 1, 0.0, 1, 1, 1, 6, 3, 20),
    ("hubo", 48, 4, 2, 0.0, 1, 1, 1, 6, 3, 20),
    ("hubo_real", 40, 6, 1, 0.02, 1, 1, 0, 4, 2, 16),
]


@pytest.mark.parametrize("kind,n,P,K,eps,spb,wls,cls,probes,csweeps,steps", OPT_CASES)
def test_run_optimal_bit_exact(oracle, kind, n, P, K, eps, spb, wls, cls, probes, csweeps, steps):
    model = make(kind, n, 61)
    om = oracle_model(oracle, model)
    beta, js, je, alpha, rf, rs = 2.0, 0.05, 2.0, 15.0 / 14.0, 0.3, 0.1
    reads, seed = 3, 515
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors([1.0], [1.0]), P, K)
    res = ann.run_optimal_reads(beta, js, je, eps, alpha, steps, spb, wls, cls, probes, csweeps, rf, rs,
                                reads=reads, seed=seed)
    for r in range(reads):
        o = oracle.sqa_opt_run(om, P, K, beta, js, je, eps, alpha, steps, spb, wls, cls, probes, csweeps, rf, rs,
                               seed, r)
        np.testing.assert_array_equal(res[r].best_state.as_array(), o["best"])
        if kind in REAL_KINDS:
            assert res[r].best_energy == pytest.approx(oracle.energy64(om, o["best"]), rel=1e-12, abs=1e-12)
        else:
            assert res[r].best_energy == o["best_energy"]
        np.testing.assert_array_equal(np.asarray(res[r].energy_trace), o["trace"])
        np.testing.assert_array_equal(np.asarray(res[r].j_perp_trace), o["j_perp"])
        np.testing.assert_array_equal(np.asarray(res[r].chi_B_trace), o["chi"])
        sc = o["scalars"]
        assert (res[r].calibrated_eps_tilde, res[r].j_perp_start, res[r].resolved_j_perp_end,
                res[r].final_j_perp) == (sc[0], sc[1], sc[2], sc[3])
    # the schedule moves: J_perp rises from j_perp_start towards j_perp_end
    jt = np.asarray(res[0].j_perp_trace)
    assert jt[-1] > js and jt[-1] <= je + 1e-12


def test_run_optimal_rotated_bit_exact(oracle, monkeypatch):
    """More rings than SMs: the phases with >= 200 sweeps run as rotated
    launches of ring groups; every read equals the oracle's."""
    model = make("dense", 40, 61)
    om = oracle_model(oracle, model)
    P, K, eps, spb, wls, cls, probes, csweeps, steps = 4, 2, 0.0, 2, 1, 0, 6, 3, 120
    beta, js, je, alpha, rf, rs = 2.0, 0.05, 2.0, 15.0 / 14.0, 0.3, 0.1
    reads, seed = 80, 717
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors([1.0], [1.0]), P, K)
    args = (beta, js, je, eps, alpha, steps, spb, wls, cls, probes, csweeps, rf, rs)
    res = ann.run_optimal_reads(*args, reads=reads, seed=seed)
    rotated = ann.last_stats.sweep_launches
    with monkeypatch.context() as mp:
        mp.setenv("QA_WHOLE_GRID", "1")
        whole = ann.run_optimal_reads(*args, reads=reads, seed=seed)
        whole_launches = ann.last_stats.sweep_launches
    # the rotated run issued ring-group launches that the whole-grid run did not
    assert rotated > whole_launches, (rotated, whole_launches)
    for r in range(reads):
        np.testing.assert_array_equal(res[r].best_state.as_array(), whole[r].best_state.as_array())
        assert res[r].best_energy == whole[r].best_energy
    for r in range(reads):
        o = oracle.sqa_opt_run(om, P, K, beta, js, je, eps, alpha, steps, spb, wls, cls, probes, csweeps, rf, rs,
                               seed, r)
        np.testing.assert_array_equal(res[r].best_state.as_array(), o["best"])
        assert res[r].best_energy == o["best_energy"]
        np.testing.assert_array_equal(np.asarray(res[r].energy_trace), o["trace"])
        np.testing.assert_array_equal(np.asarray(res[r].j_perp_trace), o["j_perp"])
        np.testing.assert_array_equal(np.asarray(res[r].chi_B_trace), o["chi"])


def test_run_optimal_single_read_and_csv(oracle, tmp_path):
    """run_optimal() after set_seed(s + r) reproduces read r of a batch; the
    diagnostic CSV holds one row per step."""
    h, J = sk_dense(40, 5)
    model = qa.DenseIsing(h, J)
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors([1.0], [1.0]), 8, 1)
    batch = ann.run_optimal_reads(1.5, 0.1, 1.5, 0.0, num_steps=20, sweeps_per_step=1, calib_probes=4,
                                  calib_sweeps=2, reads=3, seed=40)
    ann.set_seed(42)
    path = os.path.join(tmp_path, "opt.csv")
    one = ann.run_optimal(1.5, 0.1, 1.5, 0.0, num_steps=20, sweeps_per_step=1, calib_probes=4, calib_sweeps=2,
                          debug_csv_path=path)
    np.testing.assert_array_equal(one.best_state.as_array(), batch[2].best_state.as_array())
    assert one.best_energy == batch[2].best_energy
    assert one.j_perp_trace == batch[2].j_perp_trace
    with open(path) as f:
        rows = f.read().strip().splitlines()
    assert len(rows) == 21 and rows[0].startswith("phase,")


def test_run_optimal_argument_errors():
    h, J = sk_dense(8, 1)
    ann = qa.SQAAnnealer(qa.DenseIsing(h, J), qa.SQASchedule.from_vectors([1.0], [1.0]), 4, 1)
    with pytest.raises(ValueError):
        ann.run_optimal(1.0, 0.5, 0.5, 0.0)
    with pytest.raises(ValueError):
        ann.run_optimal(1.0, 0.1, 1.0, 0.0, num_steps=0)
    with pytest.raises(ValueError):
        ann.run_optimal(1.0, 0.1, 1.0, 0.0, sweeps_per_step=0)
    big = qa.SQAAnnealer(qa.DenseIsing(h, J), qa.SQASchedule.from_vectors([1.0], [1.0]), 65, 1)
    with pytest.raises(NotImplementedError):
        big.run_optimal(1.0, 0.1, 1.0, 0.0, num_steps=4, cluster_sweeps=1)


def test_solve_optimal_sqa():
    """solve(method='sqa', schedule_type='optimal') (solver.py:616-702)."""
    h, J = sk_dense(40, 3)
    d = qa.DenseIsing(h, J)
    kw = dict(trotter_slices=8, sweeps_per_beta=2, worldline_sweeps=1, optimal_num_steps=30, optimal_calib_probes=4,
              optimal_calib_sweeps=2)
    r = qa.solve(d, method="sqa", schedule_type="optimal", reads=4, seed=11, **kw)
    assert len(r.samples) == 4 and r.best_energy == min(r.energies)
    assert r.best_energy == pytest.approx(d.energy(r.best_sample), abs=1e-9)
    assert len(r.trace) == 30
    one = qa.solve(d, method="sqa", schedule_type="optimal", reads=1, seed=12, **kw)
    assert one.energies[0] == r.energies[1]


PTOPT_CASES = [
    # kind, n, rungs, P, sweeps/step, worldline, cluster, steps, swap interval, eps_tilde, J_end, continuous slices
    ("dense", 64, 4, 8, 2, 1, 0, 24, 1, 0.0, 2.0, 0),
    ("dense", 48, 3, 16, 1, 1, 1, 20, 2, 0.0, 2.5, 0),
    ("dense", 40, 3, 4, 1, 0, 0, 12, 1, 0.0, 0.0, 10),
    ("dense", 40, 3, 8, 0, 2, 0, 12, 1, 0.05, 2.0, 0),
    ("dense", 40, 3, 8, 1, 0, 0, 10, 1, 0.0, 0.5, 0),
    ("dense_h", 70, 4, 6, 1, 0, 0, 18, 3, 0.03, 2.0, 0),
    ("sparse", 128, 4, 8, 1, 1, 0, 20, 1, 0.0, 0.0, 0),
    ("sparse_real", 96, 3, 6, 1, 1, 1, 16, 2, 0.02, 2.0, 0),
    ("hubo", 48, 3, 4, 1, 1, 1, 16, 2, 0.0, 2.0, 0),
    ("hubo_real", 40, 3, 6, 1, 0, 0, 14, 1, 0.0, 2.0, 0),
]


@pytest.mark.parametrize("kind,n,R,P,spb,wls,cls,steps,swap,eps,je,cts", PTOPT_CASES)
def test_sqapt_run_optimal_bit_exact(oracle, kind, n, R, P, spb, wls, cls, steps, swap, eps, je, cts):
    """SQAParallelTemperingAnnealer.run_optimal (sqa_parallel_tempering.cpp:348-882)
    on the GPU equals the oracle: best and final states, traces, J_perp and chi_B."""
    model = make(kind, n, 67)
    om = oracle_model(oracle, model)
    betas, gammas = np.geomspace(0.5, 3.0, R), np.geomspace(2.0, 0.3, R)
    alpha, probes, csweeps = 15.0 / 14.0, 5, 3
    reads, seed = 3, 919
    ann = qa.SQAParallelTemperingAnnealer(model, betas, gammas, P)
    res = ann.run_optimal_reads(steps, spb, wls, eps, alpha, je, cls, swap, cts, probes, csweeps, reads=reads,
                                seed=seed)
    Pr = cts if cts > P else P
    swaps = 0.0
    for r in range(reads):
        o = oracle.sqapt_opt_run(om, betas, gammas, Pr, spb, wls, cls, steps, swap, eps, alpha, je, probes, csweeps,
                                 seed, r)
        np.testing.assert_array_equal(res[r].best_state.as_array(), o["best"])
        if kind in REAL_KINDS:
            assert res[r].best_energy == pytest.approx(oracle.energy64(om, o["best"]), rel=1e-12, abs=1e-12)
        else:
            assert res[r].best_energy == o["best_energy"]
        np.testing.assert_array_equal(np.asarray(res[r].final_energies), o["final_E"])
        for k in range(R):
            np.testing.assert_array_equal(res[r].final_states[k].as_array(), o["final_spins"][k])
        np.testing.assert_array_equal(np.asarray(res[r].average_energy_trace), o["avg"])
        np.testing.assert_array_equal(np.asarray(res[r].swap_acceptance_trace), o["swap"])
        np.testing.assert_array_equal(np.asarray(res[r].j_perp_trace), o["j_perp"])
        np.testing.assert_array_equal(np.asarray(res[r].chi_B_trace), o["chi"])
        sc = o["scalars"]
        assert (res[r].calibrated_eps_tilde, res[r].j_perp_start, res[r].resolved_j_perp_end,
                res[r].final_j_perp) == (sc[0], sc[1], sc[2], sc[3])
        swaps += float(np.sum(o["swap"]))
    if kind == "dense":
        assert swaps > 0.0  # the SK ladders exchange rungs; the other instances need not


def test_sqapt_run_optimal_rotated_bit_exact(oracle, monkeypatch):
    """More rings than SMs: segments with >= 8 sweeps run as rotated launches
    joined before the swaps; every read equals the oracle's."""
    model = make("dense", 48, 67)
    om = oracle_model(oracle, model)
    R, P, spb, wls, cls, steps, swap, eps, je, cts = 4, 4, 2, 1, 0, 24, 6, 0.0, 2.0, 0
    betas, gammas = np.geomspace(0.5, 3.0, R), np.geomspace(2.0, 0.3, R)
    alpha, probes, csweeps, reads, seed = 15.0 / 14.0, 5, 3, 40, 929
    ann = qa.SQAParallelTemperingAnnealer(model, betas, gammas, P)
    args = (steps, spb, wls, eps, alpha, je, cls, swap, cts, probes, csweeps)
    res = ann.run_optimal_reads(*args, reads=reads, seed=seed)
    rotated = ann.last_stats.sweep_launches
    with monkeypatch.context() as mp:
        mp.setenv("QA_WHOLE_GRID", "1")
        ann.run_optimal_reads(*args, reads=reads, seed=seed)
        whole_launches = ann.last_stats.sweep_launches
    assert rotated > whole_launches, (rotated, whole_launches)  # ring groups, not whole-grid launches
    for r in range(reads):
        o = oracle.sqapt_opt_run(om, betas, gammas, P, spb, wls, cls, steps, swap, eps, alpha, je, probes, csweeps,
                                 seed, r)
        np.testing.assert_array_equal(res[r].best_state.as_array(), o["best"])
        assert res[r].best_energy == o["best_energy"]
        np.testing.assert_array_equal(np.asarray(res[r].final_energies), o["final_E"])
        np.testing.assert_array_equal(np.asarray(res[r].average_energy_trace), o["avg"])
        np.testing.assert_array_equal(np.asarray(res[r].swap_acceptance_trace), o["swap"])
        np.testing.assert_array_equal(np.asarray(res[r].j_perp_trace), o["j_perp"])


def test_sqapt_run_optimal_errors_and_solve():
    h, J = sk_dense(30, 2)
    d = qa.DenseIsing(h, J)
    ann = qa.SQAParallelTemperingAnnealer(d, [0.5, 2.0], [2.0, 0.5], 4)
    with pytest.raises(ValueError):
        ann.run_optimal(0, 1)
    with pytest.raises(ValueError):
        ann.run_optimal(5, 1, swap_interval=0)
    with pytest.raises(ValueError):
        ann.run_optimal(5, 0, 0, cluster_sweeps=0)
    with pytest.raises(NotImplementedError):
        qa.SQAParallelTemperingAnnealer(d, [0.5, 2.0], [2.0, 0.5], 65).run_optimal(4, 1, cluster_sweeps=1)
    kw = dict(trotter_slices=8, sweeps_per_beta=1, worldline_sweeps=1, replicas=3, optimal_num_steps=20,
              optimal_calib_probes=4, optimal_calib_sweeps=2)
    r = qa.solve(d, method="sqapt", schedule_type="optimal", reads=3, seed=5, **kw)
    assert r.best_energy == min(r.energies) and len(r.trace) == 20
    assert r.best_energy == pytest.approx(d.energy(r.best_sample), abs=1e-9)
    one = qa.solve(d, method="sqapt", schedule_type="optimal", reads=1, seed=7, **kw)
    assert one.energies[0] == r.energies[2]
