"""The launch-shape autotuner: every shape it can choose leaves the results
bit for bit those of the oracle (warps per ring, the +-1 kernel's ring-state
forms, rotated launches with their step counts and group sizes), and a tuned
cache entry is applied to later runs of its bucket."""
import ctypes as C
import json
import os

import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200 import _lib, autotune
from test_gpu_parity_sa_sqa import make, oracle_model

pytestmark = pytest.mark.gpu

SHAPES = [
    dict(warps_per_ring=1), dict(warps_per_ring=3), dict(warps_per_ring=32),
    dict(field_form=0), dict(field_form=1), dict(field_form=2),
    dict(rotate=0), dict(rotate=1, rot_steps=1, rot_group=3), dict(rotate=1, rot_steps=7, rot_group=2),
]


@pytest.mark.parametrize("order", ["reference", "checkerboard"])
@pytest.mark.parametrize("kind,n,P", [("dense", 96, 8), ("sparse", 80, 6), ("dense_int", 50, 5)])
def test_every_shape_is_bit_exact(oracle, kind, n, P, order):
    model = make(kind, n, 21)
    om = oracle_model(oracle, model)
    betas, gammas = np.full(9, 0.25 * P), np.linspace(2.5, 0.1, 9)
    reads, seed = 160, 55  # more rings than SMs: rotated launches can run
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(betas, gammas), P, 1)
    eng = _lib.Engine.get(None)
    qa.set_update_order(order)
    oracle.set_update_order(order)
    want = [oracle.sqa_run(om, betas, gammas, P, 1, 1, 1, seed, r) for r in (0, 77, 159)]
    try:
        for shape in SHAPES:
            autotune.set_tuning(eng, shape)
            res = ann.run_reads(1, 1, reads=reads, seed=seed)
            for r, w in zip((0, 77, 159), want):
                np.testing.assert_array_equal(res[r].best_state.as_array(), w[0], err_msg=str(shape))
                np.testing.assert_array_equal(np.asarray(res[r].energy_trace), w[2], err_msg=str(shape))
    finally:
        autotune.set_tuning(eng, None)
        qa.set_update_order("reference")
        oracle.set_update_order("reference")


def test_tune_and_apply_cache(tmp_path):
    path = os.path.join(tmp_path, "tune.json")
    model = make("dense", 128, 4)
    betas, gammas = np.full(40, 4.0), np.linspace(3.0, 0.05, 40)
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(betas, gammas), 16, 1)
    entry = autotune.tune_sqa(ann, 1, 1, reads=200, timing_steps=40, cache_path=path)
    assert entry["ms"] <= entry["auto_ms"] and len(entry["candidates"]) > 4
    data = json.load(open(path))
    key = autotune.bucket("dense", 128, 16, 200)
    assert key in data
    base = ann.run_reads(1, 1, reads=200, seed=3)
    autotune.use_cache(path)
    try:
        tuned = ann.run_reads(1, 1, reads=200, seed=3)
        eng = _lib.Engine.get(None)
        t = _lib.qa_tuning()
        _lib.check(eng.L.qa_get_tuning(eng.h, C.byref(t)))
        assert {k: getattr(t, k) for k in autotune.AUTO} == {**autotune.AUTO, **data[key]["tuning"]}
    finally:
        autotune.use_cache(None)
        autotune.set_tuning(_lib.Engine.get(None), None)
    for a, b in zip(base, tuned):
        assert a.best_energy == b.best_energy and a.energy_trace == b.energy_trace


def test_chi_shapes_bit_exact_and_tune(tmp_path):
    """SQA-Chi under every launch shape (pilot and production; more rings than
    SMs and >= 200 production sweeps, so rotated launches can run) returns the
    automatic shape's reads bit for bit; tune_chi caches an entry in the
    SQA-Chi bucket and later runs apply it with the same results."""
    model = make("dense", 40, 43)
    P, K, steps, spb, points, sweeps, burn = 4, 2, 30, 8, 5, 6, 2
    beta, g0, g1, reads, seed = 0.4 * P, 3.0, 0.05, 80, 2468
    ann = qa.SQAChiAnnealer(model, P, K)
    eng = _lib.Engine.get(None)
    args = (beta, g0, g1, steps, spb, points, sweeps, burn)
    want = ann.run_chi_reads(*args, reads=reads, seed=seed)
    try:
        for shape in SHAPES:
            autotune.set_tuning(eng, shape)
            got = ann.run_chi_reads(*args, reads=reads, seed=seed)
            for a, b in zip(want, got):
                assert a.best_energy == b.best_energy, shape
                np.testing.assert_array_equal(a.best_state.as_array(), b.best_state.as_array(), err_msg=str(shape))
                np.testing.assert_array_equal(np.asarray(a.energy_trace), np.asarray(b.energy_trace),
                                              err_msg=str(shape))
    finally:
        autotune.set_tuning(eng, None)
    path = os.path.join(tmp_path, "tune.json")
    entry = autotune.tune_chi(ann, reads, cache_path=path, seed=seed, beta=beta, gamma_start=g0, gamma_end=g1,
                              num_steps=steps, sweeps_per_step=spb, scan_points=points, scan_sweeps=sweeps,
                              scan_burn=burn)
    assert entry["ms"] <= entry["auto_ms"] and len(entry["candidates"]) > 4
    assert autotune.bucket("dense-chi", 40, P, reads * K) in json.load(open(path))
    autotune.use_cache(path)
    try:
        got = ann.run_chi_reads(*args, reads=reads, seed=seed)
    finally:
        autotune.use_cache(None)
        autotune.set_tuning(eng, None)
    for a, b in zip(want, got):
        assert a.best_energy == b.best_energy
        np.testing.assert_array_equal(np.asarray(a.energy_trace), np.asarray(b.energy_trace))
