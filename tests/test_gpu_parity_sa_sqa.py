"""Bit-exact parity of the CUDA SA / SQA engine against the CPU restatement.

Every case calls the engine through the C ABI (libqa_gpu.so via the package's
annealer classes) and the oracle (oracle/qa_oracle.c) on the same seeded
instance and key.  With integer couplings every quantity is exact, so best
spins, best energies and the whole energy trace must agree bit for bit.
"""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200.instances import geometric_betas, hubo_random, regular3, sk_dense

pytestmark = pytest.mark.gpu


def oracle_model(oracle, model):
    if isinstance(model, qa.DenseIsing):
        return oracle.dense(model.fields(), model.couplings(), model.constant())
    if isinstance(model, qa.SparseIsing):
        e = [(x.i, x.j, x.value) for x in model.edges()]
        return oracle.sparse(model.size(), model._h, e, model.constant())
    terms = [(k, v) for k, v in model.terms()] + [((i,), hv) for i, hv in enumerate(model.h()) if hv != 0.0]
    return oracle.hubo(model.size(), terms, model.constant())


def make(kind, n, seed):
    if kind == "dense":
        h, J = sk_dense(n, seed)
        return qa.DenseIsing(h, J)
    if kind == "dense_h":
        rng = np.random.default_rng(seed + 7)
        h, J = sk_dense(n, seed)
        h = rng.choice([-0.5, 0.0, 0.25, 0.5], size=n)
        return qa.DenseIsing(h, J, 1.5)
    if kind == "dense_hwide":
        # fields whose float64 sums round (h spans 2^-100 .. 2^3): energies summed, not tracked
        rng = np.random.default_rng(seed + 9)
        h, J = sk_dense(n, seed)
        h = rng.normal(0.0, 2.0, size=n)
        h[::7] = 1e-30
        return qa.DenseIsing(h, J)
    if kind == "dense_int":
        rng = np.random.default_rng(seed)
        J = np.triu(rng.choice([-2.0, -1.0, 1.0, 2.0], size=(n, n)), 1)
        return qa.DenseIsing(rng.choice([-1.0, 0.0, 1.0], size=n), J + J.T)
    if kind == "sparse":
        h, e = regular3(n, seed)
        return qa.SparseIsing(h, e, n, -2.0)
    if kind == "sparse_deg6":
        # rows of up to six neighbours, couplings in {-2, -1, 1, 2}: integer
        # couplings whose rows do not fit the 16-byte neighbour records, so the
        # on-demand-field kernel reads its CSR rows
        h, e1 = regular3(n, seed)
        _, e2 = regular3(n, seed + 1)
        rng = np.random.default_rng(seed + 5)
        return qa.SparseIsing(h, [(a, b, w * float(rng.choice([1.0, 2.0]))) for a, b, w in e1 + e2], n, 0.0)
    if kind == "sparse_real":
        h, e = regular3(n, seed)
        rng = np.random.default_rng(seed + 3)
        return qa.SparseIsing(h, [(a, b, float(w) * rng.uniform(0.2, 1.3)) for a, b, w in e], n, 0.5)
    if kind == "hubo":
        return qa.HigherOrderIsing(hubo_random(n, seed, integer=True), n)
    if kind == "hubo_real":
        return qa.HigherOrderIsing(hubo_random(n, seed, integer=False), n)
    if kind == "hubo_deg5":
        rng = np.random.default_rng(seed)
        terms = {tuple(sorted(rng.choice(n, size=5, replace=False).tolist())): 1.0 for _ in range(n)}
        terms.update({tuple(sorted(rng.choice(n, size=2, replace=False).tolist())): -1.0 for _ in range(n)})
        return qa.HigherOrderIsing(terms, n)
    raise ValueError(kind)


def _check_best_energy(oracle, om, kind, res, E_track, best):
    """Integer couplings: the reported energy equals the tracked one bit for
    bit.  Real couplings: the tracked energy uses the float32 couplings the
    sweep runs on, the reported one is recomputed in float64 from the given
    coefficients (as qanneal reports it); compare that with the oracle's
    float64 energy of the same state."""
    if kind in REAL_KINDS:
        assert res.best_energy == pytest.approx(oracle.energy64(om, best), rel=1e-12, abs=1e-12)
    else:
        assert res.best_energy == E_track


REAL_KINDS = ("hubo_real", "sparse_real", "dense_hwide")

SA_CASES = [("dense", 64), ("dense", 100), ("dense", 256), ("dense_h", 96), ("sparse", 128), ("sparse", 70),
            ("hubo", 60), ("hubo_real", 64), ("hubo_deg5", 40)]


@pytest.mark.parametrize("kind,n", SA_CASES)
def test_sa_bit_exact(oracle, kind, n):
    model = make(kind, n, 11)
    om = oracle_model(oracle, model)
    betas = geometric_betas(0.1, 5.0, 30)
    reads, spb, seed = 6, 4, 12345
    ann = qa.Annealer(model, qa.AnnealSchedule.from_betas(betas))
    res = ann.run_reads(spb, reads=reads, seed=seed)
    tot_acc = 0
    for r in range(reads):
        best, E, trace, cnt = oracle.sa_run(om, betas, spb, seed, r)
        tot_acc += cnt[1]
        np.testing.assert_array_equal(res[r].best_state.as_array(), best)
        _check_best_energy(oracle, om, kind, res[r], E, best)
        np.testing.assert_array_equal(np.asarray(res[r].energy_trace), trace)
        assert res[r].best_energy == pytest.approx(model.energy(res[r].best_state.spins), abs=1e-9)
    st = ann.last_stats
    assert st.slice_attempts == reads * len(betas) * spb * n
    assert st.slice_accepts == tot_acc


SQA_CASES = [
    # +-1 dense couplings run on the bit-packed kernel (ring_pm1_kernel)
    ("dense", 64, 8, 1, 1, 1, 1.0),
    ("dense", 96, 5, 2, 1, 1, 1.0),
    ("dense", 40, 1, 1, 2, 0, 1.0),
    ("dense", 40, 2, 3, 0, 2, 1.0),
    ("dense", 512, 32, 1, 1, 1, 2.0),
    ("dense", 100, 64, 1, 1, 2, 0.25),
    ("dense", 33, 3, 1, 2, 3, 0.1),
    ("dense", 256, 16, 1, 0, 3, 0.05),  # many accepted worldline moves
    ("dense_h", 70, 6, 2, 2, 1, 0.5),
    ("dense_hwide", 96, 8, 1, 1, 1, 0.5),
    # rings too large for int32 fields: int16 fields with J bits in shared
    # memory (n=1024, P=32), then with J read from L2 (the rest)
    ("dense", 1024, 32, 1, 1, 1, 1.0),
    ("dense", 1024, 64, 1, 1, 1, 0.5),
    ("dense_h", 1500, 20, 1, 1, 1, 0.5),
    ("dense", 2048, 8, 1, 1, 2, 0.5),
    # the generic field-cache kernel
    ("dense_int", 80, 8, 2, 1, 1, 0.5),
    ("sparse", 128, 8, 1, 1, 1, 1.0),
    ("sparse", 64, 7, 2, 2, 1, 1.0),
    ("sparse", 2048, 16, 1, 1, 2, 0.5),  # integer couplings: on-demand fields
    ("sparse", 150, 64, 1, 1, 1, 1.0),
    ("sparse_deg6", 96, 8, 1, 1, 1, 1.0),  # integer couplings in CSR rows
    ("sparse", 96, 8, 1, 0, 3, 0.1),  # many accepted worldline moves, neighbours in one block
    ("sparse_real", 96, 6, 1, 1, 1, 1.0),  # real couplings: the field cache
    ("hubo", 48, 4, 2, 1, 1, 1.0),
    # real couplings: field updates in the same float order as the oracle's
    ("hubo_real", 64, 6, 1, 2, 1, 1.0),
    # a degree-5 term: the term-by-term update path
    ("hubo_deg5", 40, 4, 1, 1, 1, 1.0),
]


@pytest.mark.parametrize("kind,n,P,K,spb,wls,bscale", SQA_CASES)
def test_sqa_bit_exact(oracle, kind, n, P, K, spb, wls, bscale):
    _sqa_case(oracle, kind, n, P, K, spb, wls, bscale)


@pytest.mark.parametrize("kind,n,P,K,spb,wls,bscale", [("dense", 64, 8, 2, 1, 1, 1.0), ("dense", 200, 16, 1, 1, 1, 0.3)])
def test_sqa_generic_kernel_on_pm1_models(oracle, monkeypatch, kind, n, P, K, spb, wls, bscale):
    """The generic field-cache kernel gives the same bits as the +-1 kernel."""
    monkeypatch.setenv("QA_DISABLE_PM1", "1")
    _sqa_case(oracle, kind, n, P, K, spb, wls, bscale)


def test_sqa_pm1_int32_only_falls_back(oracle, monkeypatch):
    """A +-1 ring too large for int32 fields in shared memory (n=1024, P=32)
    runs on the generic kernel under QA_PM1_INT32_ONLY, with the same bits."""
    monkeypatch.setenv("QA_PM1_INT32_ONLY", "1")
    _sqa_case(oracle, "dense", 1024, 32, 1, 1, 1, 1.0)


@pytest.mark.parametrize("kind,n,P,K,spb,wls,bscale", [("sparse", 128, 8, 1, 1, 1, 1.0), ("sparse", 64, 7, 2, 2, 1, 1.0)])
def test_sqa_cached_field_kernel_on_integer_sparse(oracle, monkeypatch, kind, n, P, K, spb, wls, bscale):
    """The field-cache kernel gives the same bits as the on-demand one."""
    monkeypatch.setenv("QA_DISABLE_SPARSE_INT", "1")
    _sqa_case(oracle, kind, n, P, K, spb, wls, bscale)


CLUSTER_CASES = [
    # kind, n, P, K, spb, wls, cluster sweeps, beta scale
    ("dense", 64, 8, 2, 1, 1, 1, 1.0),
    ("dense", 40, 1, 1, 1, 0, 2, 1.0),
    ("dense", 40, 2, 1, 0, 1, 2, 1.0),
    ("dense", 33, 5, 1, 1, 0, 1, 0.5),
    ("dense", 100, 64, 1, 0, 1, 1, 0.25),
    ("dense_h", 70, 6, 2, 0, 0, 3, 0.5),
    ("dense_int", 48, 12, 1, 1, 1, 1, 0.5),
    ("sparse", 128, 8, 1, 1, 1, 1, 1.0),
    ("sparse_real", 96, 6, 1, 0, 1, 2, 1.0),
    ("hubo", 48, 4, 2, 1, 1, 1, 1.0),
    ("hubo_real", 64, 6, 1, 1, 0, 1, 1.0),
]


@pytest.mark.parametrize("kind,n,P,K,spb,wls,cls,bscale", CLUSTER_CASES)
def test_sqa_cluster_bit_exact(oracle, kind, n, P, K, spb, wls, cls, bscale):
    """Imaginary-time cluster moves (sqa_annealer.cpp:215-288) on the GPU equal the oracle's."""
    _sqa_case(oracle, kind, n, P, K, spb, wls, bscale, cls)


def _sqa_case(oracle, kind, n, P, K, spb, wls, bscale, cls=0):
    model = make(kind, n, 21)
    om = oracle_model(oracle, model)
    steps = 25
    betas = np.full(steps, bscale * 2.0 * P / 4.0)
    gammas = np.linspace(3.0, 0.05, steps)
    reads, seed = 3, 777
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(betas, gammas), P, K)
    res = ann.run_reads(spb, wls, cls, reads=reads, seed=seed)
    acc_s = acc_w = 0
    for r in range(reads):
        best, E, trace, cnt = oracle.sqa_run(om, betas, gammas, P, K, spb, wls, seed, r, cls=cls)
        acc_s += cnt[1]
        acc_w += cnt[3]
        np.testing.assert_array_equal(res[r].best_state.as_array(), best)
        _check_best_energy(oracle, om, kind, res[r], E, best)
        np.testing.assert_array_equal(np.asarray(res[r].energy_trace), trace)
    st = ann.last_stats
    assert st.slice_attempts == reads * K * P * steps * spb * n
    assert st.worldline_attempts == reads * K * steps * wls * n
    assert st.slice_accepts == acc_s and st.worldline_accepts == acc_w


@pytest.mark.parametrize("kind,n,P,K,reads", [("dense", 40, 4, 1, 160), ("dense_h", 33, 6, 2, 80),
                                               ("sparse", 64, 4, 1, 150), ("hubo", 24, 4, 1, 152),
                                               ("dense", 36, 4, 1, 151),    # a last group of one ring
                                               ("sparse", 48, 4, 1, 300)])  # groups of 3 rings
def test_sqa_rotated_launches_bit_exact(oracle, kind, n, P, K, reads):
    """More rings than SMs and >= 200 steps: the rings run as groups on side
    streams in short launches; every read equals the oracle's."""
    model = make(kind, n, 23)
    om = oracle_model(oracle, model)
    steps = 210
    betas = np.full(steps, 0.6 * P)
    gammas = np.linspace(2.5, 0.05, steps)
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(betas, gammas), P, K)
    res = ann.run_reads(1, 1, reads=reads, seed=4242)
    assert ann.last_stats.sweep_launches > (steps + 255) // 256  # not one whole-grid launch per segment
    acc_s = acc_w = 0
    for r in range(reads):
        best, E, trace, cnt = oracle.sqa_run(om, betas, gammas, P, K, 1, 1, 4242, r)
        acc_s += cnt[1]
        acc_w += cnt[3]
        np.testing.assert_array_equal(res[r].best_state.as_array(), best)
        _check_best_energy(oracle, om, kind, res[r], E, best)
        np.testing.assert_array_equal(np.asarray(res[r].energy_trace), trace)
    st = ann.last_stats
    assert st.slice_attempts == reads * K * P * steps * n
    assert st.slice_accepts == acc_s and st.worldline_accepts == acc_w


def test_single_run_matches_batch(oracle):
    """run() after set_seed(s + r) reproduces read r of a batch seeded s (solve()'s seeding)."""
    model = make("dense", 64, 3)
    sched = qa.SQASchedule.from_vectors([2.0] * 10, np.linspace(2.0, 0.1, 10))
    ann = qa.SQAAnnealer(model, sched, 4, 1)
    batch = ann.run_reads(1, 1, reads=3, seed=99)
    for r in range(3):
        ann.set_seed(99 + r)
        one = ann.run(1, 1)
        np.testing.assert_array_equal(one.best_state.as_array(), batch[r].best_state.as_array())
        assert one.best_energy == batch[r].best_energy


def test_reference_sqa_basic():
    """tests/test_sqa_basic.cpp: n=3, P=8, K=2, trace length and best energy consistency."""
    h = np.zeros(3)
    J = np.array([[0.0, 0.5, -0.3], [0.5, 0.0, 0.2], [-0.3, 0.2, 0.0]])
    ham = qa.DenseIsing(h, J)
    sched = qa.SQASchedule.from_vectors([0.2, 0.5, 1.0], [2.0, 1.0, 0.5])
    ann = qa.SQAAnnealer(ham, sched, 8, 2)
    ann.set_seed(42)
    res = ann.run(5, 1)
    assert len(res.energy_trace) == 3
    assert abs(ham.energy(res.best_state.spins) - res.best_energy) < 1e-12


def test_real_couplings_energy(oracle):
    """Real-valued J: every returned energy equals the float64 energy of its state."""
    from qlatanneal_b200.instances import dense_real
    h, J = dense_real(80, 5)
    model = qa.DenseIsing(h, J, 0.25)
    om = oracle.dense(h, J, 0.25)
    sa = qa.Annealer(model, qa.AnnealSchedule.from_betas(geometric_betas(0.1, 5.0, 20)))
    for r in sa.run_reads(3, reads=8, seed=5):
        E64 = oracle.energy64(om, r.best_state.as_array())
        assert r.best_energy == pytest.approx(E64, rel=1e-12, abs=1e-12)
    sq = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors([3.0] * 12, np.linspace(2.0, 0.1, 12)), 6, 2)
    for r in sq.run_reads(1, 1, reads=4, seed=9):
        E64 = oracle.energy64(om, r.best_state.as_array())
        assert r.best_energy == pytest.approx(E64, rel=1e-12, abs=1e-12)


def test_argument_errors():
    h, J = sk_dense(16, 1)
    m = qa.DenseIsing(h, J)
    with pytest.raises(ValueError):
        qa.Annealer(m, qa.AnnealSchedule.from_betas([1.0])).run(0)
    with pytest.raises(ValueError):
        qa.SQAAnnealer(m, qa.SQASchedule.from_vectors([1.0], [1.0]), 4).run(0, 0)
    with pytest.raises(NotImplementedError):  # cluster moves keep a slice's worldline in 64 bits
        qa.SQAAnnealer(m, qa.SQASchedule.from_vectors([1.0], [1.0]), 65).run(1, 1, cluster_sweeps=1)
