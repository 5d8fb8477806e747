"""qanneal's observers (observer.hpp, sqa_observer.hpp, metrics_observer.hpp:13-193).

The GPU sweep kernels write a strided trace into a device buffer during the run
(``qa_sa_trace_run`` / ``qa_sqa_trace_run``); after the run the engine calls the
observer's ``record`` / ``record_sweep`` in the order the reference's loops
call them (annealer.cpp:48-71, sqa_annealer.cpp:318-473).  Any object with
those methods works as an observer; a ``stride`` attribute (>= 1) limits which
sweeps the kernels record.  SQA states are passed as int8 arrays of shape
(replicas, slices, n).
"""
from __future__ import annotations

from typing import List

import numpy as np


def magnetization(spins) -> float:
    """Mean spin (metrics.hpp:11-24)."""
    s = np.asarray(spins.as_array() if hasattr(spins, "as_array") else spins)
    return float(int(s.astype(np.int64).sum()) / s.size) if s.size else 0.0


class Observer:
    """``qanneal.Observer``: ``record(step, beta, energy, state)`` once per step."""

    def record(self, step: int, beta: float, energy: float, state) -> None:
        pass


class SweepObserver:
    """``record_sweep(step, sweep, beta, energy, state)`` after each sweep."""

    def record_sweep(self, step: int, sweep: int, beta: float, energy: float, state) -> None:
        pass


class MetricsObserver(Observer):
    """Energy and magnetisation per step (metrics_observer.hpp:13-32)."""

    def __init__(self):
        self.energy_trace: List[float] = []
        self.magnetization_trace: List[float] = []

    def record(self, step, beta, energy, state):
        self.energy_trace.append(float(energy))
        self.magnetization_trace.append(magnetization(state))

    def clear(self):
        self.energy_trace.clear()
        self.magnetization_trace.clear()


class StateTraceObserver(Observer, SweepObserver):
    """Every ``stride``-th sweep's state (metrics_observer.hpp:72-110)."""

    def __init__(self):
        self.stride = 1
        self.step_trace: List[int] = []
        self.sweep_trace: List[int] = []
        self.beta_trace: List[float] = []
        self.energy_trace: List[float] = []
        self.state_trace: List[List[int]] = []

    def record_sweep(self, step, sweep, beta, energy, state):
        if self.stride > 1 and sweep % self.stride != 0:
            return
        self.step_trace.append(int(step))
        self.sweep_trace.append(int(sweep))
        self.beta_trace.append(float(beta))
        self.energy_trace.append(float(energy))
        self.state_trace.append(state.spins)

    def clear(self):
        for t in (self.step_trace, self.sweep_trace, self.beta_trace, self.energy_trace, self.state_trace):
            t.clear()


class SQAObserver:
    """``qanneal.SQAObserver``: ``record(step, beta, gamma, avg_energy, state)`` once per step."""

    def record(self, step: int, beta: float, gamma: float, avg_energy: float, state: np.ndarray) -> None:
        pass


class SQASweepObserver:
    """``record_sweep(step, replica, sweep, phase, beta, gamma, avg_energy,
    replica_energies, state)`` after each sweep of each replica; phase 0 slice,
    1 worldline, 2 cluster (sqa_observer.hpp:22-26)."""

    def record_sweep(self, step, replica, sweep, phase, beta, gamma, avg_energy, replica_energies, state) -> None:
        pass


class SQAMetricsObserver(SQAObserver):
    """Average energy and magnetisation over replicas and slices per step
    (metrics_observer.hpp:34-70)."""

    def __init__(self):
        self.energy_trace: List[float] = []
        self.magnetization_trace: List[float] = []

    def record(self, step, beta, gamma, avg_energy, state):
        self.energy_trace.append(float(avg_energy))
        self.magnetization_trace.append(magnetization(state))

    def clear(self):
        self.energy_trace.clear()
        self.magnetization_trace.clear()


class SQAStateTraceObserver(SQAObserver, SQASweepObserver):
    """Every ``stride``-th sweep of every replica: the full state, the average
    and per-replica energies (metrics_observer.hpp:112-190)."""

    def __init__(self):
        self.stride = 1
        self.replicas = self.slices = self.spins = 0
        self.step_trace: List[int] = []
        self.replica_trace: List[int] = []
        self.sweep_trace: List[int] = []
        self.phase_trace: List[int] = []
        self.beta_trace: List[float] = []
        self.gamma_trace: List[float] = []
        self.avg_energy_trace: List[float] = []
        self.replica_energy_trace: List[List[float]] = []
        self.state_trace: List[List[int]] = []

    def record_sweep(self, step, replica, sweep, phase, beta, gamma, avg_energy, replica_energies, state):
        if self.stride > 1 and sweep % self.stride != 0:
            return
        if self.replicas == 0:
            self.replicas, self.slices, self.spins = (int(x) for x in state.shape)
        self.step_trace.append(int(step))
        self.replica_trace.append(int(replica))
        self.sweep_trace.append(int(sweep))
        self.phase_trace.append(int(phase))
        self.beta_trace.append(float(beta))
        self.gamma_trace.append(float(gamma))
        self.avg_energy_trace.append(float(avg_energy))
        self.replica_energy_trace.append([float(e) for e in replica_energies])
        self.state_trace.append(state.reshape(-1).astype(int).tolist())

    def clear(self):
        self.replicas = self.slices = self.spins = 0
        for t in (self.step_trace, self.replica_trace, self.sweep_trace, self.phase_trace, self.beta_trace,
                  self.gamma_trace, self.avg_energy_trace, self.replica_energy_trace, self.state_trace):
            t.clear()


def observer_stride(observer) -> int:
    return max(int(getattr(observer, "stride", 1) or 1), 1)


def replay_sa(observer, betas, spb: int, stride: int, trace, energies, states, step_states, State) -> None:
    """The reference's call order: record_sweep after each sweep, record at each step end."""
    sweep_obs = hasattr(observer, "record_sweep")
    step_obs = hasattr(observer, "record")
    for step, beta in enumerate(betas):
        if sweep_obs:
            for k, sw in enumerate(range(0, spb, stride)):
                observer.record_sweep(step, sw, float(beta), float(energies[step, k]), State(states[step, k]))
        if step_obs:
            observer.record(step, float(beta), float(trace[step]), State(step_states[step]))


def replay_sqa(observer, betas, gammas, P: int, K: int, spb: int, cls: int, wls: int, stride: int, trace,
               ring_states, ring_E, step_states, step_E) -> None:
    """record_sweep for each recorded sweep of each replica (replicas in turn,
    slice, cluster, worldline sweeps), then record at the step end.  A sweep
    record holds the replicas before it at this step's end, the replica itself
    after the sweep, the replicas after it at the previous step's end; energies
    are summed slice by slice and replica by replica as the reference does."""
    sweep_obs = hasattr(observer, "record_sweep")
    step_obs = hasattr(observer, "record")
    ns, nc = -(-spb // stride), -(-cls // stride)
    phases = ((0, spb, 0), (2, cls, ns), (1, wls, ns + nc))

    def ring_sum(E) -> float:
        s = 0.0
        for e in E:
            s += float(e)
        return s

    for step in range(len(betas)):
        beta, gamma = float(betas[step]), float(gammas[step])
        if sweep_obs:
            for r in range(K):
                for phase, count, off in phases:
                    for sw in range(0, count, stride):
                        idx = off + sw // stride
                        sums, parts = [], []
                        for k in range(K):
                            if k < r:
                                st, E = step_states[k, step + 1], step_E[k, step + 1]
                            elif k == r:
                                st, E = ring_states[k, step, idx], ring_E[k, step, idx]
                            else:
                                st, E = step_states[k, step], step_E[k, step]
                            parts.append(st)
                            sums.append(ring_sum(E))
                        total = 0.0
                        for x in sums:
                            total += x
                        observer.record_sweep(step, r, sw, phase, beta, gamma, total / (K * P),
                                              [x / P for x in sums], np.stack(parts))
        if step_obs:
            observer.record(step, beta, gamma, float(trace[step]), step_states[:, step + 1].copy())
