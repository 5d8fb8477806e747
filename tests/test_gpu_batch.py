"""Several models of one kind in one launch (BatchRunner over the multi-problem
C ABI): model p's reads equal its own single-model run with the same seed."""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200.instances import geometric_betas
from test_gpu_parity_sa_sqa import make

pytestmark = pytest.mark.gpu

KIND_SIZES = [("dense", (40, 64, 97)), ("sparse", (64, 130, 96)), ("hubo", (33, 48, 40)), ("dense_h", (70, 31, 128))]


def _same(a, b, fields):
    for f in fields:
        x, y = getattr(a, f), getattr(b, f)
        if hasattr(x, "as_array"):
            np.testing.assert_array_equal(x.as_array(), y.as_array())
        else:
            np.testing.assert_array_equal(np.asarray(x), np.asarray(y))


@pytest.mark.parametrize("kind,sizes", KIND_SIZES)
def test_batch_equals_single_runs(kind, sizes):
    models = [make(kind, n, 100 + i) for i, n in enumerate(sizes)]
    runner = qa.BatchRunner()
    betas = geometric_betas(0.1, 3.0, 10)
    sa = runner.anneal(models, qa.AnnealSchedule.from_betas(betas), 2, reads=3, seed=41)
    sched = qa.SQASchedule.from_vectors(np.full(8, 3.0), np.linspace(2.5, 0.1, 8))
    sqa = runner.sqa(models, sched, 6, 2, 1, 1, 1, reads=2, seed=43)
    pb, pg = np.geomspace(0.3, 3.0, 3), np.geomspace(2.0, 0.3, 3)
    pt = runner.sqapt(models, pb, pg, 4, 1, 1, 6, 2, reads=2, seed=47)
    for p, m in enumerate(models):
        one = qa.Annealer(m, qa.AnnealSchedule.from_betas(betas)).run_reads(2, reads=3, seed=41)
        for a, b in zip(sa[p], one):
            _same(a, b, ("best_state", "best_energy", "energy_trace"))
        one = qa.SQAAnnealer(m, sched, 6, 2).run_reads(1, 1, 1, reads=2, seed=43)
        for a, b in zip(sqa[p], one):
            _same(a, b, ("best_state", "best_energy", "energy_trace"))
        one = qa.SQAParallelTemperingAnnealer(m, pb, pg, 4).run_reads(1, 1, 6, 2, reads=2, seed=47)
        for a, b in zip(pt[p], one):
            _same(a, b, ("best_state", "best_energy", "average_energy_trace", "swap_acceptance_trace",
                         "final_energies"))
            for x, y in zip(a.final_states, b.final_states):
                np.testing.assert_array_equal(x.as_array(), y.as_array())


def test_batch_rejects_mixed_kinds():
    with pytest.raises(ValueError):
        qa.BatchRunner().anneal([make("dense", 16, 1), make("sparse", 16, 2)],
                                qa.AnnealSchedule.from_betas([1.0]), 1)
    with pytest.raises(ValueError):
        qa.BatchRunner().anneal([], qa.AnnealSchedule.from_betas([1.0]), 1)


def test_sharded_instance_set_single_rank_equals_batch(tmp_path):
    """run_instances_sharded with its default runner (BatchRunner) on a
    one-rank group: the same per-instance results as the batched call."""
    import torch.distributed as dist
    from qlatanneal_b200.distributed import run_instances_sharded
    from qlatanneal_b200.instances import sk_dense
    models = [qa.DenseIsing(*sk_dense(n, 300 + n)) for n in (40, 72, 24)]
    betas, gammas = np.full(8, 2.0), np.linspace(2.0, 0.1, 8)
    sched = qa.SQASchedule.from_vectors(betas, gammas)
    dist.init_process_group("gloo", init_method=f"file://{tmp_path}/pg", rank=0, world_size=1)
    try:
        res = run_instances_sharded("sqa", models, reads=4, seed=9, schedule=sched, trotter_slices=8,
                                    sweeps_per_beta=1, worldline_sweeps=1)
    finally:
        dist.destroy_process_group()
    want = qa.BatchRunner().sqa(models, sched, 8, sweeps_per_beta=1, worldline_sweeps=1, reads=4, seed=9)
    assert res.plan == [[0, 1, 2]]
    for i, reads in enumerate(want):
        es = [r.best_energy for r in reads]
        k = min(range(len(es)), key=lambda q: (es[q], q))
        assert res.best_energy[i] == es[k] and res.best_read[i] == k
        np.testing.assert_array_equal(res.best_state[i], reads[k].best_state.as_array())
