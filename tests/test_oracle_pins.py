"""Pins the CPU restatement (the oracle) before any GPU result is trusted.

* Philox4x32-10 against the published Random123 known-answer vectors.
* The deterministic exp of the Metropolis test against math.exp.
* Model functions against the reference's own golden tests
  (tests/test_dense_ising.cpp, tests/test_higher_order_ising.cpp) and against
  qanneal compiled from its sources (oracle/_ref).
* SA / SQA restatements against the unmodified reference, statistically.
"""
import math

import numpy as np
import pytest

from qlatanneal_b200.instances import geometric_betas, hubo_random, regular3, sk_dense

# Random123 kat_vectors, philox4x32 with 10 rounds: (counter, key, expected)
PHILOX_KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(oracle, ctr, key, want):
    assert oracle.philox(ctr, key).tolist() == want


def test_det_exp_accuracy(oracle):
    ys = np.linspace(-16.999, 0.0, 20001).astype(np.float32)
    for y in ys[::7]:
        got = oracle.expf(float(y))
        assert abs(got - math.exp(float(y))) <= 1.5e-6 * math.exp(float(y))
    assert oracle.expf(0.0) == 1.0


def test_dense_ising_golden(oracle, ref):
    """tests/test_dense_ising.cpp: n=2, h=(1,-1), J01=0.5: E(+1,+1)=0.5, dE matches a flip."""
    h = np.array([1.0, -1.0])
    J = np.array([[0.0, 0.5], [0.5, 0.0]])
    m = oracle.dense(h, J)
    s = np.array([1, 1], np.int8)
    assert oracle.energy64(m, s) == 0.5
    assert ref.dense(h, J).energy(s) == 0.5
    s2 = s.copy()
    s2[0] = -1
    assert abs((oracle.energy64(m, s2) - 0.5) - oracle.delta_energy64(m, s, 0)) < 1e-12


def _brute(s, h, terms, c):
    E = c + float(np.dot(h, s))
    for vars_, cf in terms:
        E += cf * float(np.prod(s[list(vars_)]))
    return E


def _random_hubo(n, rng):
    """tests/test_higher_order_ising.cpp:64-85: degrees 1-4, repeated indices,
    duplicated supports and a fully cancelling term."""
    terms = []
    for _ in range(40):
        d = int(rng.integers(1, 5))
        terms.append(([int(v) for v in rng.integers(0, n, d)], float(rng.uniform(-1.5, 1.5))))
    terms += [([0, 1, 2], 0.7), ([2, 1, 0], -0.3), ([3, 3, 4, 4], 9.9)]
    h = np.zeros(n)
    return h, terms, float(rng.uniform(-1.5, 1.5))


@pytest.mark.parametrize("n", [5, 8, 12, 20])
def test_hubo_brute_force(oracle, ref, n):
    rng = np.random.default_rng(0xC0FFEE + n)
    for rep in range(3):
        h, terms, c = _random_hubo(n, rng)
        m = oracle.hubo(n, terms, c)
        rm = ref.hubo(n, terms, c)
        T, _, c_ref, h_ref = rm.hubo_info()
        tptr, tvars, coef, h_or, c_or = oracle.hubo_terms(m)
        assert len(coef) == T and c_or == c_ref
        np.testing.assert_array_equal(h_or, h_ref)
        for _ in range(30):
            s = rng.choice([-1, 1], n).astype(np.int8)
            E = oracle.energy64(m, s)
            assert abs(E - _brute(s.astype(float), h, terms, c)) < 1e-9
            assert E == rm.energy(s)
            for f in range(n):
                s2 = s.copy()
                s2[f] = -s2[f]
                de = oracle.delta_energy64(m, s, f)
                assert abs(de - (_brute(s2.astype(float), h, terms, c) - E)) < 1e-9
                assert de == rm.delta_energy(s, f)
            # float32 field cache gives the float64 delta to float32 accuracy
            g = oracle.fields(m, s)
            np.testing.assert_allclose(g.astype(np.float64), rm.fields(s) - h_ref, rtol=1e-6, atol=1e-5)


def test_dense_sparse_energies_match_reference(oracle, ref):
    rng = np.random.default_rng(3)
    h, J = sk_dense(50, 4, h_sigma=0.1)
    m, rm = oracle.dense(h, J), ref.dense(h, J)
    hs, edges = regular3(64, 5)
    ms, rms = oracle.sparse(64, hs, edges + [(0, 1, 0.5), (1, 0, -0.25)], 0.75), \
        ref.sparse(64, hs, edges + [(0, 1, 0.5), (1, 0, -0.25)], 0.75)
    for _ in range(20):
        s = rng.choice([-1, 1], 50).astype(np.int8)
        assert oracle.energy64(m, s) == rm.energy(s)
        assert oracle.delta_energy64(m, s, 7) == rm.delta_energy(s, 7)
        s = rng.choice([-1, 1], 64).astype(np.int8)
        assert oracle.energy64(ms, s) == rms.energy(s)
        assert oracle.delta_energy64(ms, s, 0) == pytest.approx(rms.delta_energy(s, 0), abs=1e-12)


def test_tracking_energy_exact_for_integer_models(oracle):
    rng = np.random.default_rng(9)
    h, J = sk_dense(96, 2)
    h = rng.choice([-0.5, 0.0, 0.5], 96)
    m = oracle.dense(h, J, 3.0)
    hs, edges = regular3(80, 1)
    ms = oracle.sparse(80, hs, edges, -1.0)
    mh = oracle.hubo(40, list(hubo_random(40, 3, integer=True).items()), 0.5)
    for mod, n in ((m, 96), (ms, 80), (mh, 40)):
        for _ in range(10):
            s = rng.choice([-1, 1], n).astype(np.int8)
            assert oracle.energy_track(mod, s) == oracle.energy64(mod, s)


def _diff_z(a, b):
    """|mean(a) - mean(b)| in standard errors of the difference."""
    a, b = np.asarray(a, float), np.asarray(b, float)
    se = math.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
    d = abs(a.mean() - b.mean())
    if se == 0.0:
        return 0.0 if d <= 1e-12 else math.inf
    return d / se


def _agree(sample, reads):
    """sample(reads, stage) -> [(oracle values, reference values), ...] of one
    configuration.  Every statistic's means must lie within the combined 95%
    interval of the difference; a configuration that misses is drawn once more
    with fresh seeds (stage 1) and four times the reads, and must then agree
    within the combined 99% interval: a chance miss rarely repeats, a real
    bias persists with the added power.  Seeds are fixed, so the outcome is
    too."""
    z1 = [_diff_z(a, b) for a, b in sample(reads, 0)]
    if max(z1) <= 1.96:
        return
    z2 = [_diff_z(a, b) for a, b in sample(4 * reads, 1)]
    assert max(z2) <= 2.576, (z1, z2)


# seeds of the second stage start this far from the first's
STAGE = 1_000_003


def test_sa_restatement_matches_reference_statistics(oracle, ref):
    """The replay-model SA and qanneal's Annealer sample the same distribution
    of best energies (means within the combined 95% interval, 400 reads each)."""
    h, J = sk_dense(48, 5)
    m, rm = oracle.dense(h, J), ref.dense(h, J)
    betas = geometric_betas(0.1, 2.0, 12)

    def sample(R, st):
        eo = [oracle.sa_run(m, betas, 2, 1000 + st * STAGE, k)[1] for k in range(R)]
        er = [rm.sa_run(betas, 2, 5000 + st * STAGE + k)[1] for k in range(R)]
        return [(eo, er)]
    _agree(sample, 400)


def test_sqapt_restatement_matches_reference_statistics(oracle, ref):
    """Replay-model SQA-PT vs qanneal's SQAParallelTemperingAnnealer: final
    average projected energy and mean swap acceptance agree (combined 95%
    interval)."""
    h, J = sk_dense(24, 7)
    m, rm = oracle.dense(h, J), ref.dense(h, J)
    betas = np.geomspace(0.3, 3.0, 4)
    gammas = np.linspace(2.0, 0.1, 4)
    P, steps = 6, 8

    def sample(R, st):
        eo, er, so, sr = [], [], [], []
        for k in range(R):
            o = oracle.sqapt_run(m, betas, gammas, P, 1, 1, steps, 2, 100 + st * STAGE, k)
            r = rm.sqapt_run(betas, gammas, P, 1, 1, steps, 2, 7000 + st * STAGE + k)
            eo.append(o[4][-1]); er.append(r[3][-1]); so.append(o[5].sum()); sr.append(r[4].sum())
        return [(eo, er), (so, sr)]
    _agree(sample, 250)


def test_sqa_restatement_matches_reference_statistics(oracle, ref):
    h, J = sk_dense(32, 6)
    m, rm = oracle.dense(h, J), ref.dense(h, J)
    steps, P, K = 10, 8, 1
    betas = np.full(steps, 1.5)
    gammas = np.linspace(2.0, 0.2, steps)

    def sample(R, st):
        eo = [oracle.sqa_run(m, betas, gammas, P, K, 1, 1, 1000 + st * STAGE, k)[2][-1] for k in range(R)]
        er = [rm.sqa_run(betas, gammas, P, K, 1, 1, 9000 + st * STAGE + k)[2][-1] for k in range(R)]
        return [(eo, er)]
    _agree(sample, 300)


def test_cluster_sqa_restatement_matches_reference_statistics(oracle, ref):
    """Imaginary-time cluster moves (sqa_annealer.cpp:215-288) alone, at fixed
    (beta, Gamma): the replay form and qanneal's SQAAnnealer reach the same
    average energy (mean of the last 50 steps, 300 reads each, inside the
    combined 95% CI).  The reference's acceptance adds the boundary Trotter
    term on top of the bond probabilities, so its move does not keep the
    Trotter action's distribution and the stationary state depends on the
    other moves' order; cluster-only dynamics is where the two must agree."""
    h, J = sk_dense(12, 11)
    m, rm = oracle.dense(h, J), ref.dense(h, J)
    steps, P = 100, 4
    for beta, gamma in ((0.5, 1.0), (2.0, 2.0)):
        b, g = np.full(steps, beta), np.full(steps, gamma)

        def sample(R, st):
            eo = [oracle.sqa_run(m, b, g, P, 1, 0, 0, 100 + st * STAGE, k, cls=1)[2][-50:].mean() for k in range(R)]
            er = [rm.sqa_run(b, g, P, 1, 0, 0, 7000 + st * STAGE + k, cls=1)[2][-50:].mean() for k in range(R)]
            return [(eo, er)]
        _agree(sample, 300)
        mo = np.mean(sample(50, 0)[0][0])
        start = [oracle.sqa_run(m, b[:1], g[:1], P, 1, 0, 0, 100, k, cls=1)[2][0] for k in range(50)]
        assert mo < np.mean(start) - 1.0  # the moves do anneal


def test_cluster_sqapt_restatement_matches_reference_statistics(oracle, ref):
    h, J = sk_dense(20, 11)
    m, rm = oracle.dense(h, J), ref.dense(h, J)
    betas = np.geomspace(0.5, 3.0, 3)
    gammas = np.linspace(1.5, 0.2, 3)
    P, steps = 6, 80

    def sample(R, st):
        eo = [oracle.sqapt_run(m, betas, gammas, P, 0, 0, steps, 2, 100 + st * STAGE, k, cls=2)[4][-20:].mean()
              for k in range(R)]
        er = [rm.sqapt_run(betas, gammas, P, 0, 0, steps, 2, 7000 + st * STAGE + k, cls=2)[3][-20:].mean()
              for k in range(R)]
        return [(eo, er)]
    _agree(sample, 300)


def test_classical_pt_restatement_matches_reference_statistics(oracle, ref):
    """Classical parallel tempering (parallel_tempering.cpp:36-122): at
    equilibrium the replay form and qanneal's ParallelTemperingAnnealer have
    the same average energy and swap acceptance (combined 95% interval, 300 reads)."""
    h, J = sk_dense(20, 13)
    m, rm = oracle.dense(h, J), ref.dense(h, J)
    betas = np.geomspace(0.2, 2.0, 4)
    steps = 60

    def sample(R, st):
        eo, er, so, sr = [], [], [], []
        for k in range(R):
            o = oracle.pt_run(m, betas, 1, steps, 2, 100 + st * STAGE, k)
            r = rm.pt_run(betas, 1, steps, 2, 7000 + st * STAGE + k)
            eo.append(o[4][-20:].mean()); er.append(r[3][-20:].mean())
            so.append(o[5][1::2].mean()); sr.append(r[4][1::2].mean())
        return [(eo, er), (so, sr)]
    _agree(sample, 300)


def test_replica_restatement_matches_reference_statistics(oracle, ref):
    """ReplicaAnnealer (replica_annealer.cpp:46-142) is independent SA
    replicas; its average energy and magnetisation traces match qanneal's."""
    rng = np.random.default_rng(3)
    h, J = sk_dense(24, 14)
    h = rng.choice([0.5, 1.0, 0.0], size=24)
    m, rm = oracle.dense(h, J), ref.dense(h, J)
    betas = geometric_betas(0.1, 2.0, 10)
    R = 8

    def sample(N, st):
        eo, mo, er, mr = [], [], [], []
        for k in range(N):
            runs = [oracle.replica_run(m, betas, 2, 500 + st * STAGE + 100 * k, r) for r in range(R)]
            eo.append(np.mean([x[2][-1] for x in runs])); mo.append(np.mean([x[3][-1] for x in runs]))
            _, avg, mag = rm.replica_run(betas, 2, R, 9000 + st * STAGE + k)
            er.append(avg[-1]); mr.append(mag[-1])
        return [(eo, er), (mo, mr)]
    _agree(sample, 60)


@pytest.mark.parametrize("eps", [0.0, 0.02])
def test_run_optimal_restatement_matches_reference_statistics(oracle, ref, eps):
    """SQAAnnealer::run_optimal (sqa_annealer.cpp:499-952): beta ramp,
    calibration pilot (eps_tilde <= 0) or online J_perp updates (eps_tilde > 0),
    chi_B from bond-sum samples.  Final energy, the J_perp reached mid-run and
    the calibrated budget agree with qanneal (combined 95% interval, 200 reads)."""
    h, J = sk_dense(24, 17)
    m, rm = oracle.dense(h, J), ref.dense(h, J)
    a = (8, 2, 2.0, 0.05, 2.0, eps, 15 / 14, 30, 2, 1, 1, 8, 4, 0.3, 0.1)
    fs = (lambda d: d["trace"][-1], lambda d: d["j_perp"][20], lambda d: d["scalars"][0],
          lambda d: d["best_energy"])

    def sample(R, st):
        A = [oracle.sqa_opt_run(m, *a, seed=100 + st * STAGE, read=k) for k in range(R)]
        B = [rm.sqa_opt_run(*a, seed=5000 + st * STAGE + k) for k in range(R)]
        return [([f(d) for d in A], [f(d) for d in B]) for f in fs]
    _agree(sample, 200)
    d = oracle.sqa_opt_run(m, *a, seed=100, read=0)
    assert d["scalars"][1] == 0.05 and d["scalars"][2] == 2.0
    assert np.all(np.diff(d["j_perp"][9:]) >= 0) and d["j_perp"][-1] <= 2.0 + 1e-12


@pytest.mark.parametrize("eps,je", [(0.0, 2.0), (0.03, 2.0), (0.0, 0.0)])
def test_sqapt_run_optimal_restatement_matches_reference_statistics(oracle, ref, eps, je):
    """SQAParallelTemperingAnnealer::run_optimal (sqa_parallel_tempering.cpp:348-882):
    one J_perp shared by every rung, calibration from the starting states
    (eps_tilde <= 0) or online updates (eps_tilde > 0), classical swaps.  The
    final rung energies, J_perp mid-run, the calibrated budget, the best energy
    and the swap rate agree with qanneal (combined 95% interval, 150 reads); J_end = 0
    resolves to the coldest rung's coupling."""
    h, J = sk_dense(20, 23)
    m, rm = oracle.dense(h, J), ref.dense(h, J)
    betas, gammas = np.geomspace(0.5, 3.0, 4), np.geomspace(2.0, 0.3, 4)
    a = (betas, gammas, 6, 2, 1, 1, 24, 2, eps, 15 / 14, je, 6, 3)
    d = oracle.sqapt_opt_run(m, *a, seed=300, read=0)
    b = a
    if je <= 0.0:
        # the sentinel resolves to the coldest rung's coupling; the reference is
        # handed that value (its warning for the sentinel, written through
        # std::cerr, does not survive being loaded through ctypes here)
        je = 0.5 * np.log(1.0 / np.tanh(betas[-1] * gammas[-1] / 6))
        assert d["scalars"][2] == pytest.approx(je, rel=1e-14)
        b = a[:10] + (je,) + a[11:]
    fs = (lambda x: x["avg"][-1], lambda x: x["final_E"][-1], lambda x: x["j_perp"][12],
          lambda x: x["scalars"][0], lambda x: x["best_energy"], lambda x: np.mean(x["swap"][1::2]))

    def sample(R, st):
        A = [oracle.sqapt_opt_run(m, *a, seed=300 + st * STAGE, read=k) for k in range(R)]
        B = [rm.sqapt_opt_run(*b, seed=7000 + st * STAGE + k) for k in range(R)]
        return [([f(x) for x in A], [f(x) for x in B]) for f in fs]
    _agree(sample, 150)
    # the resolved J range is deterministic
    B0 = rm.sqapt_opt_run(*b, seed=7000)
    for k in (1, 2):
        assert d["scalars"][k] == pytest.approx(B0["scalars"][k], rel=1e-15)
    assert np.all(np.diff(d["j_perp"]) >= 0) and d["j_perp"][-1] <= d["scalars"][2] + 1e-12
    assert np.all(d["swap"][0::2] == 0.0)
