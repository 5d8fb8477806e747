"""Learned chi_B-curve MLP: oracle self-checks (CPU), CUDA gradients and Adam
against the float64 oracle, training on pilot curves, and what the trained
network gains over the plain pilot scan in SQA-Chi (GPU)."""
import os
import sys
import time

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import mlp_oracle as mo  # noqa: E402

DIMS = [16, 128, 128, 128, 128]


def _rand_params(dims, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k, n in zip(dims[:-1], dims[1:]):
        out.append(rng.uniform(-1, 1, k * n) * np.sqrt(6.0 / k))
        out.append(rng.normal(0, 0.1, n))
    return np.concatenate(out)


# ---------------------------------------------------------------- CPU
def test_oracle_backprop_matches_finite_differences():
    dims = [5, 7, 6, 4]
    rng = np.random.default_rng(3)
    p = _rand_params(dims, 4)
    X = rng.normal(size=(9, 5))
    T = rng.normal(size=(9, 2))
    _, g = mo.loss_and_grads(p, dims, X, T, bf16=False)
    idx = rng.choice(p.size, 40, replace=False)
    fd = mo.finite_difference(p, dims, X, T, idx)
    assert np.max(np.abs(fd - g[idx]) / (np.abs(g[idx]) + 1e-8)) < 1e-5


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.00390625, 1.005859375, -3.14159, 0.0, 65504.0], np.float32)
    want = np.array([1.0, 1.0, 1.0078125, -3.140625, 0.0, 65536.0], np.float32)
    assert np.array_equal(mo.bf16_round(x), want)


def test_features_and_targets():
    from qlatanneal_b200.instances import regular3, sk_dense
    from qlatanneal_b200.learned import N_FEATURES, curve_target, instance_features, target_curve
    from qlatanneal_b200.models import DenseIsing, SparseIsing

    h, J = sk_dense(64, 5)
    fd = instance_features(DenseIsing(h, J), 4.0, 3.0, 0.01, 16)
    h2, e = regular3(64, 5)
    fs = instance_features(SparseIsing(h2, e, 64), 4.0, 3.0, 0.01, 16)
    assert fd.shape == (N_FEATURES,) and fs.shape == (N_FEATURES,)
    assert np.all(np.isfinite(fd)) and np.all(np.isfinite(fs))
    # SK: top eigenvalue ~ 2 sqrt(n) J_rms (semicircle edge); 3-regular +-1: <= 3
    assert 1.6 < fd[10] < 2.3 and fs[10] <= 3.0 / np.sqrt(3.0) + 1e-9
    assert abs(fd[1] - 63 / 64) < 1e-12 and abs(fs[1] - 3 / 64) < 1e-12
    chi = np.abs(np.sin(np.linspace(0, 3, 64))) * 5
    assert np.allclose(target_curve(curve_target(chi)), chi / chi.max(), atol=1e-12)


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_gpu_gradients_match_oracle():
    from qlatanneal_b200.learned import ChiCurveModel

    m = ChiCurveModel(seed=11)
    p = _rand_params(DIMS, 12).astype(np.float32)
    m.set_params(p)
    assert np.array_equal(m.get_params(), p)
    rng = np.random.default_rng(13)
    for B in (1, 37, 256):
        X = rng.normal(size=(B, 16)).astype(np.float32)
        T = rng.normal(size=(B, 64)).astype(np.float32)
        m.mu, m.sd = np.zeros(16), np.ones(16)
        loss, g = m.loss_grad(X, T)
        lo, go = mo.loss_and_grads(p, DIMS, X.astype(np.float64), T.astype(np.float64), bf16=True)
        assert abs(loss - lo) <= 1e-5 * abs(lo) + 1e-6
        assert np.linalg.norm(g - go) <= 2e-5 * np.linalg.norm(go)
        # layer by layer, too (a mis-indexed layer cannot hide behind the total)
        off = 0
        for k, n in zip(DIMS[:-1], DIMS[1:]):
            for cnt in (k * n, n):
                seg = slice(off, off + cnt)
                assert np.linalg.norm(g[seg] - go[seg]) <= 1e-4 * np.linalg.norm(go[seg]) + 1e-9
                off += cnt
    # forward output == oracle forward
    Y, S = m.predict(X)
    acts = mo.forward(p, DIMS, X.astype(np.float64))
    assert np.allclose(Y, acts[-1][:, :64], rtol=1e-5, atol=1e-5)


@pytest.mark.gpu
def test_gpu_adam_step_matches_oracle():
    import ctypes as C

    from qlatanneal_b200 import _lib
    from qlatanneal_b200.learned import ChiCurveModel

    m = ChiCurveModel(seed=21)
    p = m.get_params()
    rng = np.random.default_rng(22)
    X = rng.normal(size=(64, 16)).astype(np.float32)
    T = rng.normal(size=(64, 64)).astype(np.float32)
    mom, vel = np.zeros_like(p), np.zeros_like(p)
    for step in (1, 2, 3):
        _, go = mo.loss_and_grads(p, DIMS, X.astype(np.float64), T.astype(np.float64), bf16=True)
        _, g = m.loss_grad(X, T)
        loss = C.c_float()
        _lib.check(m._eng.L.qa_mlp_train_step(m._h, X.ctypes.data, T.ctypes.data, 64, C.c_float(1e-3),
                                              C.byref(loss)))
        p_ref, mom, vel = mo.adam_step(p, g, mom, vel, step, 1e-3)
        p = m.get_params()
        # the update uses the GPU's own gradient; its float32 arithmetic may differ by a few ulps
        assert np.max(np.abs(p - p_ref)) <= 1e-6
        assert np.linalg.norm(g - go) <= 2e-5 * np.linalg.norm(go)


def _instances(count, n_choices, seed):
    from qlatanneal_b200.instances import regular3, sk_dense
    from qlatanneal_b200.models import DenseIsing, SparseIsing

    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.choice(n_choices))
        s = int(rng.integers(1 << 30))
        if i % 2 == 0:
            h, J = sk_dense(n, s)
            out.append(DenseIsing(h, J))
        else:
            h, e = regular3(n, s, h_choices=(0.0,))
            out.append(SparseIsing(h, e, n))
    return out


RUN = dict(beta=4.0, gamma_start=3.0, gamma_end=0.01, slices=16)


@pytest.fixture(scope="module")
def trained():
    from qlatanneal_b200.learned import ChiCurveModel, curve_target, instance_features, pilot_curves

    train = _instances(400, [32, 48, 64, 80, 96], 101)
    chi = pilot_curves(train, RUN["beta"], RUN["gamma_start"], RUN["gamma_end"], RUN["slices"], points=64,
                       sweeps=200, burn=50, reads=4, seed=7)
    X = np.stack([instance_features(m, **RUN) for m in train])
    Y = curve_target(chi)
    model = ChiCurveModel(seed=5)
    hist = model.fit(X, Y, epochs=200, batch=64, lr=2e-3, seed=1, run_params=dict(RUN, points=64))
    return model, X, Y, hist


@pytest.mark.gpu
def test_training_fits_pilot_curves(trained):
    """Against the 16-read mean pilot curve of unseen instances, the predicted
    curve gives a schedule closer than one pilot scan's does, and it has
    learned how the two families differ."""
    from qlatanneal_b200.learned import instance_features, pilot_curves, schedule_distance, target_curve

    model, X, Y, hist = trained
    assert hist[-1] < hist[0] - 0.5
    test = _instances(24, [40, 56, 72, 88], 202)
    chi = pilot_curves(test, RUN["beta"], RUN["gamma_start"], RUN["gamma_end"], RUN["slices"], points=64,
                       sweeps=200, burn=50, reads=16, seed=9, average=False)
    truth = chi.mean(axis=1)
    mean, std = model.predict(np.stack([instance_features(m, **RUN) for m in test]))
    pred = target_curve(mean)
    d_model = float(schedule_distance(pred, truth).mean())
    d_pilot = float(schedule_distance(chi[:, 0], truth).mean())
    assert d_model < d_pilot, (d_model, d_pilot)
    dense = np.array([m.kind == "dense" for m in test])
    dp = pred[dense].mean(0) / pred[dense].mean(0).max() - pred[~dense].mean(0) / pred[~dense].mean(0).max()
    dt = truth[dense].mean(0) / truth[dense].mean(0).max() - truth[~dense].mean(0) / truth[~dense].mean(0).max()
    assert np.corrcoef(dp, dt)[0, 1] > 0.5
    assert np.all(np.isfinite(std)) and np.all(std > 0)


@pytest.mark.gpu
def test_uncertainty_falls_back_to_pilot(trained):
    from qlatanneal_b200.instances import sk_dense
    from qlatanneal_b200.models import DenseIsing

    model, *_ = trained
    assert model.max_std is not None and model.max_std > 0  # calibrated by fit()
    h, J = sk_dense(64, 77)
    m = DenseIsing(h, J)
    c = model.curve(m)
    assert c is not None and c.shape == (64,) and np.all(c >= 0) and c.max() == 1.0
    assert model.last_z <= model.max_z and model.last_std <= model.max_std
    std_m = model.last_std
    assert model.curve(m, points=16).shape == (16,)
    # an instance unlike the training set (|J| = 3): the pilot must run
    assert model.curve(DenseIsing(h, J * 3.0)) is None and model.last_z > model.max_z
    # run parameters it was not trained on
    assert model.curve(m, beta=1.0) is None
    # a predicted spread above the threshold
    keep = model.max_std
    model.max_std = 0.5 * std_m
    try:
        assert model.curve(m) is None
    finally:
        model.max_std = keep


@pytest.mark.gpu
def test_learned_schedule_beats_pilot_time_to_target(trained):
    """Same production anneal, schedule from the predicted curve vs from the
    pilot scan: the learned path reaches 99% of the best-known energy about as
    often -- its success proportion no lower than the bottom of the pilot's
    95% Wilson interval -- in less wall time (features + inference included)."""
    from qlatanneal_b200.annealers import SQAChiAnnealer

    model, *_ = trained
    test = [m for m in _instances(8, [64], 303) if m.kind == "dense"]
    reads = 32
    kw = dict(num_steps=100, sweeps_per_step=4, scan_points=64, scan_sweeps=200, scan_burn=50, reads=reads)
    t_pilot = t_learned = 0.0
    ok_pilot = ok_learned = 0
    for i, m in enumerate(test):
        ann = SQAChiAnnealer(m, RUN["slices"], 1)
        ann.run_chi_reads(RUN["beta"], RUN["gamma_start"], RUN["gamma_end"], num_steps=2, sweeps_per_step=1,
                          scan_points=4, scan_sweeps=2, scan_burn=1, reads=1, seed=1)  # warm the device copy
        t0 = time.perf_counter()
        rp = ann.run_chi_reads(RUN["beta"], RUN["gamma_start"], RUN["gamma_end"], seed=1000 + i, **kw)
        t1 = time.perf_counter()
        curve = model.curve(m)
        assert curve is not None
        rl = ann.run_chi_reads(RUN["beta"], RUN["gamma_start"], RUN["gamma_end"], seed=2000 + i, scan_chi=curve,
                               **kw)
        t2 = time.perf_counter()
        t_pilot += t1 - t0
        t_learned += t2 - t1
        ep = np.array([r.best_energy for r in rp])
        el = np.array([r.best_energy for r in rl])
        best = min(ep.min(), el.min())
        target = 0.99 * best  # best < 0 for these SK instances
        ok_pilot += int(np.sum(ep <= target))
        ok_learned += int(np.sum(el <= target))
    total = reads * len(test)
    # no loss of success probability beyond the pilot's own 95% interval
    from stats_util import wilson
    lo, _ = wilson(ok_pilot, total)
    assert ok_learned / total >= lo, (ok_learned, ok_pilot, total, lo)
    assert t_learned < t_pilot, (t_learned, t_pilot)
