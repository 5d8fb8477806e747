"""ReplicaAnnealer and classical ParallelTemperingAnnealer on the GPU against
the CPU restatement, bit for bit (replica_annealer.cpp:46-142,
parallel_tempering.cpp:36-122)."""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200.instances import geometric_betas
from test_gpu_parity_sa_sqa import REAL_KINDS, make, oracle_model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,n,R", [("dense", 64, 6), ("dense_h", 96, 4), ("sparse", 128, 5), ("hubo", 48, 3),
                                      ("hubo_real", 40, 3)])
def test_replica_annealer_bit_exact(oracle, kind, n, R):
    model = make(kind, n, 41)
    om = oracle_model(oracle, model)
    betas = geometric_betas(0.1, 4.0, 20)
    seed = 2024
    res = qa.ReplicaAnnealer(model, qa.AnnealSchedule.from_betas(betas), R).run(3, seed=seed)
    runs = [oracle.replica_run(om, betas, 3, seed, r) for r in range(R)]
    assert len(res.replicas) == R
    for r, (best, E, trace, mag, bstep) in enumerate(runs):
        rep = res.replicas[r]
        np.testing.assert_array_equal(rep.best_state.as_array(), best)
        if kind in REAL_KINDS:
            assert rep.best_energy == pytest.approx(oracle.energy64(om, best), rel=1e-12, abs=1e-12)
        else:
            assert rep.best_energy == E
        np.testing.assert_array_equal(np.asarray(rep.energy_trace), trace)
        np.testing.assert_array_equal(np.asarray(rep.magnetization_trace), mag)
    # the global best: lowest energy, first reached (earliest step, then replica)
    g = min(range(R), key=lambda r: (res.replicas[r].best_energy, runs[r][4], r))
    assert res.global_best_energy == res.replicas[g].best_energy
    np.testing.assert_array_equal(res.global_best_state.as_array(), runs[g][0])
    np.testing.assert_array_equal(np.asarray(res.average_energy_trace), np.mean([x[2] for x in runs], axis=0))
    np.testing.assert_array_equal(np.asarray(res.average_magnetization_trace),
                                  np.mean([x[3] for x in runs], axis=0))


@pytest.mark.parametrize("kind,n,R,spb,steps,swap", [("dense", 64, 4, 2, 12, 1), ("dense_int", 48, 5, 1, 9, 2),
                                                     ("sparse", 100, 6, 2, 8, 3), ("hubo", 40, 3, 1, 7, 1)])
def test_parallel_tempering_bit_exact(oracle, kind, n, R, spb, steps, swap):
    model = make(kind, n, 43)
    om = oracle_model(oracle, model)
    betas = np.geomspace(0.2, 3.0, R)
    reads, seed = 3, 4242
    res = qa.ParallelTemperingAnnealer(model, betas).run_reads(spb, steps, swap, reads=reads, seed=seed)
    swaps = 0.0
    for r in range(reads):
        best, E, fE, fs, avg, swp = oracle.pt_run(om, betas, spb, steps, swap, seed, r)
        np.testing.assert_array_equal(res[r].best_state.as_array(), best)
        assert res[r].best_energy == E
        np.testing.assert_array_equal(np.asarray(res[r].final_energies), fE)
        for k in range(R):
            np.testing.assert_array_equal(res[r].final_states[k].as_array(), fs[k])
        np.testing.assert_array_equal(np.asarray(res[r].average_energy_trace), avg)
        np.testing.assert_array_equal(np.asarray(res[r].swap_acceptance_trace), swp)
        swaps += float(np.sum(swp))
    assert swaps > 0.0


def test_argument_errors():
    from qlatanneal_b200.instances import sk_dense
    h, J = sk_dense(8, 1)
    m = qa.DenseIsing(h, J)
    with pytest.raises(ValueError):
        qa.ParallelTemperingAnnealer(m, [1.0])
    with pytest.raises(ValueError):
        qa.ParallelTemperingAnnealer(m, [1.0, 2.0]).run(0, 5)
    with pytest.raises(ValueError):
        qa.ReplicaAnnealer(m, qa.AnnealSchedule.from_betas([1.0]), 0)
    with pytest.raises(ValueError):
        qa.ReplicaAnnealer(m, qa.AnnealSchedule.from_betas([1.0]), 2).run(0)
