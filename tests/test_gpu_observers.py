"""Observers on the GPU (annealer.cpp:48-71, sqa_annealer.cpp:318-473,
metrics_observer.hpp:13-193): the sweep kernels write a strided trace into a
device buffer; the traces equal the oracle's bit for bit, the observed run
equals the unobserved one, and the observer objects are filled in the
reference's order and layout."""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200.instances import geometric_betas
from test_gpu_parity_sa_sqa import REAL_KINDS, make, oracle_model

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind,n,spb,stride", [("dense", 64, 3, 1), ("dense_h", 70, 4, 2), ("sparse", 96, 2, 1),
                                               ("hubo", 40, 3, 3), ("hubo_real", 33, 2, 1)])
def test_sa_observers_match_oracle(oracle, kind, n, spb, stride):
    model = make(kind, n, 71)
    om = oracle_model(oracle, model)
    betas = geometric_betas(0.1, 3.0, 9)
    sched = qa.AnnealSchedule.from_betas(betas)
    ann = qa.Annealer(model, sched)
    ann.set_seed(123)
    plain = ann.run(spb)
    ann.set_seed(123)
    obs = qa.StateTraceObserver()
    obs.stride = stride
    res = ann.run(spb, observer=obs)
    ann.set_seed(123)
    met = qa.MetricsObserver()
    ann.run(spb, observer=met)
    best, E, trace, states, energies, ends, mag = oracle.sa_trace_run(om, betas, spb, stride, 123, 0)
    # the observed run is the plain run
    np.testing.assert_array_equal(res.best_state.as_array(), plain.best_state.as_array())
    assert res.best_energy == plain.best_energy
    np.testing.assert_array_equal(np.asarray(res.energy_trace), trace)
    # sweep records: (step, sweep) pairs, states and energies of the oracle
    recs = [(s, w) for s in range(len(betas)) for w in range(0, spb, stride)]
    assert list(zip(obs.step_trace, obs.sweep_trace)) == recs
    assert obs.beta_trace == [float(betas[s]) for s, _ in recs]
    np.testing.assert_array_equal(np.asarray(obs.state_trace, dtype=np.int8), states.reshape(-1, n))
    assert obs.energy_trace == energies.reshape(-1).tolist()
    # per-step metrics
    assert met.energy_trace == trace.tolist()
    assert met.magnetization_trace == mag.tolist()


SQA_CASES = [
    # kind, n, P, K, spb, wls, cls, stride
    ("dense", 64, 8, 1, 2, 1, 0, 1),
    ("dense", 48, 6, 2, 2, 1, 1, 1),
    ("dense_h", 40, 5, 3, 3, 2, 0, 2),
    ("sparse", 96, 4, 2, 1, 1, 1, 1),
    ("hubo", 40, 4, 2, 1, 1, 0, 1),
    ("hubo_real", 33, 6, 1, 2, 0, 1, 1),
]


@pytest.mark.parametrize("kind,n,P,K,spb,wls,cls,stride", SQA_CASES)
def test_sqa_observers_match_oracle(oracle, kind, n, P, K, spb, wls, cls, stride):
    model = make(kind, n, 73)
    om = oracle_model(oracle, model)
    steps = 7
    betas = np.full(steps, 0.6 * P)
    gammas = np.linspace(2.5, 0.1, steps)
    ann = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(betas, gammas), P, K)
    ann.set_seed(77)
    plain = ann.run(spb, wls, cls)
    ann.set_seed(77)
    obs = qa.SQAStateTraceObserver()
    obs.stride = stride
    res = ann.run(spb, wls, cls, observer=obs)
    ann.set_seed(77)
    met = qa.SQAMetricsObserver()
    ann.run(spb, wls, cls, observer=met)
    o = oracle.sqa_trace_run(om, betas, gammas, P, K, spb, wls, cls, stride, 77, 0)
    np.testing.assert_array_equal(res.best_state.as_array(), plain.best_state.as_array())
    assert res.best_energy == plain.best_energy
    np.testing.assert_array_equal(np.asarray(res.energy_trace), o["trace"])
    assert met.energy_trace == o["trace"].tolist()
    assert met.magnetization_trace == o["mag"].tolist()
    # the sweep records assembled the way the reference's loop sees them
    ns, nc = -(-spb // stride), -(-cls // stride)
    i = 0
    for s in range(steps):
        for r in range(K):
            for phase, count, off in ((0, spb, 0), (2, cls, ns), (1, wls, ns + nc)):
                for w in range(0, count, stride):
                    idx = off + w // stride
                    assert (obs.step_trace[i], obs.replica_trace[i], obs.sweep_trace[i], obs.phase_trace[i]) == (
                        s, r, w, phase)
                    assert obs.beta_trace[i] == betas[s] and obs.gamma_trace[i] == gammas[s]
                    parts, sums = [], []
                    for k in range(K):
                        if k < r:
                            st, E = o["step_states"][k, s + 1], o["step_E"][k, s + 1]
                        elif k == r:
                            st, E = o["ring_states"][k, s, idx], o["ring_E"][k, s, idx]
                        else:
                            st, E = o["step_states"][k, s], o["step_E"][k, s]
                        parts.append(st)
                        acc = 0.0
                        for e in E:
                            acc += float(e)
                        sums.append(acc)
                    np.testing.assert_array_equal(np.asarray(obs.state_trace[i], np.int8),
                                                  np.stack(parts).reshape(-1))
                    tot = 0.0
                    for x in sums:
                        tot += x
                    assert obs.avg_energy_trace[i] == tot / (K * P)
                    assert obs.replica_energy_trace[i] == [x / P for x in sums]
                    i += 1
    assert i == len(obs.step_trace)
    assert (obs.replicas, obs.slices, obs.spins) == (K, P, n)


def test_generic_observer_objects():
    """Any object with record / record_sweep is called like the reference's observers."""
    model = make("dense", 32, 5)
    calls = []

    class Steps:
        def record(self, step, beta, energy, state):
            calls.append(("step", step, energy, state.size()))

    class Sweeps:
        stride = 2

        def record_sweep(self, step, sweep, beta, energy, state):
            calls.append(("sweep", step, sweep))

    ann = qa.Annealer(model, qa.AnnealSchedule.from_betas([0.5, 1.0, 2.0]))
    r = ann.run(3, observer=Steps())
    assert [c[1] for c in calls] == [0, 1, 2] and [c[2] for c in calls] == list(r.energy_trace)
    calls.clear()
    ann.run(3, observer=Sweeps())
    assert calls == [("sweep", s, w) for s in range(3) for w in (0, 2)]
