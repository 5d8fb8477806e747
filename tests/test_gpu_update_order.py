"""The two update orders of the SQA / SQA-PT sweeps, bit for bit against the
CPU restatement.

qanneal's order (the default) draws a fresh random spin order before every
slice, cluster and worldline sweep and sweeps the Trotter slices one after
another (sqa_annealer.cpp:181-209, 295-315; sqa_parallel_tempering.cpp:209,
224, 281); the engine runs the slices as a pipeline over blocks of visiting
positions.  The checkerboard order sweeps the slices in parity phases with
the spins ascending.  Both must equal the oracle in the same order on every
kernel form: the bit-packed +-1 kernel (int32 and int16 fields, J in shared
memory or from L2), the integer-sparse kernel and the generic kernel (dense
integer, real-valued sparse, HUBO, cluster sweeps).
"""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from test_gpu_parity_sa_sqa import REAL_KINDS, make, oracle_model

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["reference", "checkerboard"])
def order(request, oracle):
    qa.set_update_order(request.param)
    oracle.set_update_order(request.param)
    yield request.param
    qa.set_update_order("reference")
    oracle.set_update_order("reference")


SQA_CASES = [
    # kind, n, P, K, spb, wls, cls, beta
    ("dense", 64, 8, 1, 1, 1, 0, 1.0),
    ("dense", 100, 5, 2, 2, 1, 0, 1.0),
    ("dense", 33, 1, 1, 2, 1, 0, 1.0),
    ("dense", 96, 2, 1, 1, 2, 0, 0.4),
    ("dense", 200, 64, 1, 1, 1, 0, 2.0),
    ("dense_int", 70, 6, 1, 1, 1, 0, 1.0),
    ("dense_h", 96, 7, 1, 2, 1, 0, 1.0),
    ("sparse", 100, 4, 1, 2, 1, 0, 1.0),
    ("sparse", 64, 9, 2, 1, 2, 0, 0.3),
    ("sparse_deg6", 80, 6, 1, 1, 1, 0, 1.0),
    ("sparse", 96, 8, 1, 1, 3, 0, 0.15),  # many accepted worldline moves
    ("sparse_real", 80, 4, 1, 1, 1, 0, 1.0),
    ("hubo", 40, 4, 1, 1, 1, 0, 1.0),
    ("dense", 48, 6, 1, 1, 1, 1, 1.0),
    ("sparse", 60, 5, 1, 1, 0, 2, 1.0),
]


@pytest.mark.parametrize("kind,n,P,K,spb,wls,cls,beta", SQA_CASES)
def test_sqa_orders_bit_exact(oracle, order, kind, n, P, K, spb, wls, cls, beta):
    model = make(kind, n, 5)
    om = oracle_model(oracle, model)
    steps = 10
    betas = np.full(steps, beta * P / 4.0)
    gammas = np.linspace(2.5, 0.05, steps)
    reads, seed = 4, 8080
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(betas, gammas), P, K)
    res = ann.run_reads(spb, wls, cluster_sweeps=cls, reads=reads, seed=seed)
    acc = 0
    for r in range(reads):
        best, E, trace, cnt = oracle.sqa_run(om, betas, gammas, P, K, spb, wls, seed, r, cls=cls)
        np.testing.assert_array_equal(res[r].best_state.as_array(), best)
        if kind in REAL_KINDS:
            np.testing.assert_allclose(np.asarray(res[r].energy_trace), trace, rtol=1e-12, atol=1e-12)
        else:
            assert res[r].best_energy == E
            np.testing.assert_array_equal(np.asarray(res[r].energy_trace), trace)
        acc += cnt[1]
    assert ann.last_stats.slice_accepts == acc


@pytest.mark.parametrize("n,P,reads", [(512, 32, 2), (1024, 32, 1), (1500, 16, 1)])
def test_pm1_field_forms_bit_exact(oracle, order, n, P, reads):
    """int32 fields (n = 512), int16 fields with J in shared memory (n = 1024)
    and with J from L2 (n = 1500)."""
    model = make("dense", n, 9)
    om = oracle_model(oracle, model)
    steps = 4
    betas = np.full(steps, 0.5 * P)
    gammas = np.linspace(3.0, 0.5, steps)
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(betas, gammas), P, 1)
    res = ann.run_reads(1, 1, reads=reads, seed=77)
    for r in range(reads):
        best, E, trace, _ = oracle.sqa_run(om, betas, gammas, P, 1, 1, 1, 77, r)
        np.testing.assert_array_equal(res[r].best_state.as_array(), best)
        assert res[r].best_energy == E
        np.testing.assert_array_equal(np.asarray(res[r].energy_trace), trace)


@pytest.mark.parametrize("kind,n,P,R,spb,wls,cls", [("dense", 64, 8, 4, 1, 1, 0), ("sparse", 80, 4, 5, 2, 1, 0),
                                                    ("hubo", 30, 4, 3, 1, 1, 0), ("dense", 40, 6, 3, 1, 1, 1)])
def test_sqapt_orders_bit_exact(oracle, order, kind, n, P, R, spb, wls, cls):
    model = make(kind, n, 13)
    om = oracle_model(oracle, model)
    betas = np.geomspace(0.3, 3.0, R) * P / 8.0
    gammas = np.linspace(2.5, 0.05, R)
    steps, swap, reads, seed = 8, 2, 3, 4321
    ann = qa.SQAParallelTemperingAnnealer(model, betas, gammas, P)
    res = ann.run_reads(spb, wls, steps, swap, cluster_sweeps=cls, reads=reads, seed=seed)
    for r in range(reads):
        best, E, fE, fs, avg, swp, cnt = oracle.sqapt_run(om, betas, gammas, P, spb, wls, steps, swap, seed, r,
                                                          cls=cls)
        np.testing.assert_array_equal(res[r].best_state.as_array(), best)
        assert res[r].best_energy == E
        np.testing.assert_array_equal(np.asarray(res[r].final_energies), fE)
        np.testing.assert_array_equal(np.asarray(res[r].average_energy_trace), avg)
        np.testing.assert_array_equal(np.asarray(res[r].swap_acceptance_trace), swp)


def test_orders_differ_and_default_is_reference(oracle):
    """The switch changes the dynamics (same seed, different samples) and the
    default is qanneal's order."""
    assert qa.get_update_order() == "reference"
    model = make("dense", 64, 3)
    betas, gammas = np.full(6, 2.0), np.linspace(2.0, 0.1, 6)
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(betas, gammas), 8, 1)
    a = ann.run_reads(1, 1, reads=4, seed=5)
    qa.set_update_order("checkerboard")
    try:
        b = ann.run_reads(1, 1, reads=4, seed=5)
    finally:
        qa.set_update_order("reference")
    assert any(not np.array_equal(x.best_state.as_array(), y.best_state.as_array()) or
               x.energy_trace != y.energy_trace for x, y in zip(a, b))
    with pytest.raises(ValueError):
        qa.set_update_order("shuffled")
