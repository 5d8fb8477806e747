"""Host logic of the observers and of run_optimal's diagnostic CSV, on
synthetic traces (no GPU): call order, record filtering by stride, and the
assembly of an SQA sweep record from the replicas' traces (metrics_observer.hpp,
sqa_annealer.cpp:318-473)."""
import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200.annealers import SQAResult, _write_opt_debug_csv
from qlatanneal_b200.models import State
from qlatanneal_b200.observers import replay_sa, replay_sqa


class _Log:
    def __init__(self):
        self.calls = []

    def record(self, *a):
        self.calls.append(("record",) + a)

    def record_sweep(self, *a):
        self.calls.append(("sweep",) + a)


def test_replay_sa_order_and_stride():
    S, spb, stride, n = 3, 5, 2, 4
    rps = -(-spb // stride)
    energies = np.arange(S * rps, dtype=float).reshape(S, rps)
    states = np.ones((S, rps, n), np.int8)
    ends = -np.ones((S, n), np.int8)
    trace = np.array([10.0, 11.0, 12.0])
    log = _Log()
    replay_sa(log, [0.1, 0.2, 0.3], spb, stride, trace, energies, states, ends, State)
    kinds = [c[0] for c in log.calls]
    assert kinds == (["sweep"] * rps + ["record"]) * S
    sweeps = [(c[1], c[2]) for c in log.calls if c[0] == "sweep"]
    assert sweeps == [(s, w) for s in range(S) for w in (0, 2, 4)]
    assert [c[3] for c in log.calls if c[0] == "record"] == [10.0, 11.0, 12.0]
    st = qa.StateTraceObserver()
    st.stride = stride
    replay_sa(st, [0.1, 0.2, 0.3], spb, stride, trace, energies, states, ends, State)
    assert st.sweep_trace == [0, 2, 4] * S and len(st.state_trace) == S * rps
    met = qa.MetricsObserver()
    replay_sa(met, [0.1, 0.2, 0.3], spb, stride, trace, energies, states, ends, State)
    assert met.energy_trace == [10.0, 11.0, 12.0] and met.magnetization_trace == [-1.0] * S


def test_replay_sqa_assembles_replicas():
    K, P, n, S, spb, cls, wls, stride = 3, 2, 4, 2, 2, 1, 1, 1
    rps = spb + cls + wls
    ring_states = np.zeros((K, S, rps, P, n), np.int8)
    ring_E = np.zeros((K, S, rps, P))
    step_states = np.zeros((K, S + 1, P, n), np.int8)
    step_E = np.zeros((K, S + 1, P))
    # distinct values: ring k, step s, record r -> state filled with a code, energies with it too
    for k in range(K):
        for s in range(S):
            for r in range(rps):
                ring_states[k, s, r] = 1
                ring_E[k, s, r] = 100 * k + 10 * s + r
        for s in range(S + 1):
            step_states[k, s] = -1
            step_E[k, s] = -(100 * k + s)
    log = _Log()
    replay_sqa(log, [1.0, 2.0], [3.0, 4.0], P, K, spb, cls, wls, stride, [7.0, 8.0], ring_states, ring_E,
               step_states, step_E)
    sweeps = [c for c in log.calls if c[0] == "sweep"]
    assert len(sweeps) == S * K * rps
    # (step, replica, sweep, phase): slice sweeps, then cluster (2), then worldline (1)
    assert [(c[1], c[2], c[3], c[4]) for c in sweeps[:rps]] == [(0, 0, 0, 0), (0, 0, 1, 0), (0, 0, 0, 2),
                                                                 (0, 0, 0, 1)]
    # replica 1 at step 1, its first slice sweep: replica 0 at step 1's end,
    # replica 1 after the sweep, replica 2 at step 0's end
    c = next(x for x in sweeps if x[1] == 1 and x[2] == 1 and x[3] == 0 and x[4] == 0)
    state, rep_E, avg = c[9], c[8], c[7]
    assert (state[0] == -1).all() and (state[1] == 1).all() and (state[2] == -1).all()
    sums = [-(100 * 0 + 2) * P, (100 * 1 + 10 * 1 + 0) * P, -(100 * 2 + 1) * P]
    assert rep_E == [x / P for x in sums] and avg == sum(sums) / (K * P)
    records = [x for x in log.calls if x[0] == "record"]
    assert [(r[1], r[4]) for r in records] == [(0, 7.0), (1, 8.0)]
    assert records[1][5].shape == (K, P, n)


def test_sqa_state_trace_observer_fields():
    obs = qa.SQAStateTraceObserver()
    obs.stride = 2
    st = np.ones((2, 3, 4), np.int8)
    obs.record_sweep(0, 1, 1, 0, 1.0, 2.0, -3.0, [-1.0, -2.0], st)  # filtered by the stride
    obs.record_sweep(0, 1, 2, 0, 1.0, 2.0, -3.0, [-1.0, -2.0], st)
    assert (obs.replicas, obs.slices, obs.spins) == (2, 3, 4)
    assert obs.sweep_trace == [2] and obs.state_trace == [[1] * 24]
    obs.clear()
    assert obs.replicas == 0 and obs.step_trace == []


def test_opt_debug_csv(tmp_path):
    res = SQAResult(State(4), -1.0, [0.0] * 4, [0.1, 0.2, 0.4, 0.5], [2.0, 1.0, 0.5, 0.25], 0.01)
    path = tmp_path / "opt.csv"
    _write_opt_debug_csv(str(path), res, 1, 1.5)
    rows = path.read_text().strip().splitlines()
    assert rows[0].startswith("phase,step_index,j_perp,chi_B,delta_j")
    assert rows[1].startswith("beta_ramp,0,") and rows[2].startswith("run,1,")
    assert len(rows) == 5


def test_batch_runner_rejects_empty():
    with pytest.raises(ValueError):
        qa.BatchRunner().anneal([], qa.AnnealSchedule.from_betas([1.0]), 1)
