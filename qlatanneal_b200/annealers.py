"""Annealer classes with qanneal's constructor/run signatures (python/bindings.cpp:352-620).

Every ``run*`` call executes on the GPU through libqa_gpu.so.  ``run`` performs
one read, exactly like qanneal; ``run_reads`` performs many reads in a single
batched launch (the form ``solve()`` uses).  Read ``r`` of a batch seeded with
``s`` uses the same random stream as a single ``run`` after ``set_seed(s + r)``.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib, autotune
from .models import AnnealSchedule, SQASchedule, State

BACKENDS = ("cuda", "CUDA")


def _check_backend(backend: str) -> None:
    if backend in ("cpu", "CPU"):
        raise ValueError("qlatanneal_b200 implements backend='cuda' only; the CPU backend is qanneal itself.")
    if backend not in BACKENDS:
        raise ValueError("Unknown backend: " + str(backend))


def _random_seed() -> int:
    return int.from_bytes(os.urandom(8), "little")


@dataclass
class AnnealResult:
    """``qanneal.AnnealResult`` (annealer.hpp:16-20)."""
    best_state: State
    best_energy: float
    energy_trace: List[float]


@dataclass
class SQAResult:
    """``qanneal.SQAResult`` (sqa_annealer.hpp:18-29); the schedule diagnostics are filled by ``run_optimal``."""
    best_state: State
    best_energy: float
    energy_trace: List[float]
    j_perp_trace: List[float] = field(default_factory=list)
    chi_B_trace: List[float] = field(default_factory=list)
    calibrated_eps_tilde: float = 0.0
    j_perp_start: float = 0.0
    resolved_j_perp_end: float = 0.0
    final_j_perp: float = 0.0


@dataclass
class SQAParallelTemperingResult:
    """``qanneal.SQAParallelTemperingResult`` (sqa_parallel_tempering.hpp:15-29);
    the schedule diagnostics are filled by ``run_optimal``."""
    final_states: List[State]
    final_energies: List[float]
    best_state: State
    best_energy: float
    average_energy_trace: List[float]
    swap_acceptance_trace: List[float]
    j_perp_trace: List[float] = field(default_factory=list)
    chi_B_trace: List[float] = field(default_factory=list)
    calibrated_eps_tilde: float = 0.0
    j_perp_start: float = 0.0
    resolved_j_perp_end: float = 0.0
    final_j_perp: float = 0.0


@dataclass
class SQAChiResult:
    """``qanneal.SQAChiResult`` (sqa_chi_annealer.hpp:18-36)."""
    best_state: State
    best_energy: float
    energy_trace: List[float]
    beta_schedule: List[float]
    gamma_schedule: List[float]
    s_schedule: List[float]
    scan_s: List[float]
    scan_gamma: List[float]
    scan_chi_B: List[float]
    s_star: float
    gamma_star: float
    j_perp_star: float
    chi_floor: float
    driver_A0: float


@dataclass
class ReplicaResult:
    """``qanneal.ReplicaResult`` (replica_annealer.hpp:15-20)."""
    best_state: State
    best_energy: float
    energy_trace: List[float]
    magnetization_trace: List[float]


@dataclass
class MultiAnnealResult:
    """``qanneal.MultiAnnealResult`` (replica_annealer.hpp:22-28)."""
    replicas: List[ReplicaResult]
    global_best_state: State
    global_best_energy: float
    average_energy_trace: List[float]
    average_magnetization_trace: List[float]


@dataclass
class ParallelTemperingResult:
    """``qanneal.ParallelTemperingResult`` (parallel_tempering.hpp:13-20)."""
    final_states: List[State]
    final_energies: List[float]
    best_state: State
    best_energy: float
    average_energy_trace: List[float]
    swap_acceptance_trace: List[float]


def _lazy_list(name: str) -> property:
    """A result field that may be given as a numpy row and becomes a Python
    list (the reference's std::vector -> list) on first access: building
    hundreds of thousands of floats for traces nobody reads is most of the
    host time of a large batched call."""
    priv = "_lazy_" + name

    def get(self):
        v = self.__dict__[priv]
        if isinstance(v, np.ndarray):
            v = v.tolist()
            self.__dict__[priv] = v
        return v

    def set(self, v):
        self.__dict__[priv] = v

    return property(get, set)


for _cls, _names in ((AnnealResult, ("energy_trace",)), (SQAResult, ("energy_trace",)),
                     (ReplicaResult, ("energy_trace", "magnetization_trace")),
                     (MultiAnnealResult, ("average_energy_trace", "average_magnetization_trace")),
                     (ParallelTemperingResult, ("average_energy_trace", "swap_acceptance_trace")),
                     (SQAParallelTemperingResult, ("average_energy_trace", "swap_acceptance_trace")),
                     (SQAChiResult, ("energy_trace", "beta_schedule", "gamma_schedule", "s_schedule", "scan_s",
                                     "scan_gamma", "scan_chi_B"))):
    for _n in _names:
        setattr(_cls, _n, _lazy_list(_n))


@dataclass
class RunStats:
    """Device-side totals of one batched call (qa_stats)."""
    slice_attempts: int = 0
    slice_accepts: int = 0
    worldline_attempts: int = 0
    worldline_accepts: int = 0
    sweep_ms: float = 0.0
    total_ms: float = 0.0
    launches: int = 0
    sweep_launches: int = 0
    h2d_bytes: int = 0
    d2h_bytes: int = 0
    max_field_drift: float = 0.0

    @classmethod
    def from_c(cls, s: "_lib.qa_stats") -> "RunStats":
        return cls(s.slice_attempts, s.slice_accepts, s.worldline_attempts, s.worldline_accepts, s.sweep_ms,
                   s.total_ms, s.launches, s.sweep_launches, s.h2d_bytes, s.d2h_bytes, s.max_field_drift)


def set_drift_check(tolerance: float, device: Optional[int] = None) -> None:
    """Field-drift check of the incremental local-field caches (the property
    test_higher_order_ising.cpp:149-167 checks for the reference's float64
    cache): with tolerance > 0, later SA / SQA / SQA-PT runs on the device
    recompute the float32 fields in float64 after the run, report the largest
    deviation as ``last_stats.max_field_drift`` and raise
    ``FieldDriftError`` above the tolerance.  0 turns it off."""
    eng = _lib.Engine.get(device)
    _lib.check(eng.L.qa_set_drift_check(eng.h, float(tolerance)))


_ORDERS = {"reference": _lib.QA_ORDER_REFERENCE, "checkerboard": _lib.QA_ORDER_CHECKERBOARD}


def set_update_order(order: str, device: Optional[int] = None) -> None:
    """Sweep order of the SQA and SQA-PT runs on the device.

    ``"reference"`` (the default) is qanneal's: a fresh random spin order
    before every slice, cluster and worldline sweep, the Trotter slices swept
    one after another -- the engine then samples qanneal's own Markov chain,
    so its finite-time statistics match qanneal's.  ``"checkerboard"`` sweeps
    the slices in parity phases with the spins ascending (the order of
    qanneal's SQAChiAnnealer): the same stationary distribution, faster,
    different finite-time dynamics.  SQA-Chi, SA and classical parallel
    tempering keep their own orders either way."""
    if order not in _ORDERS:
        raise ValueError("update order must be 'reference' or 'checkerboard'.")
    eng = _lib.Engine.get(device)
    _lib.check(eng.L.qa_set_update_order(eng.h, _ORDERS[order]))


def get_update_order(device: Optional[int] = None) -> str:
    eng = _lib.Engine.get(device)
    v = _lib.C.c_int(0)
    _lib.check(eng.L.qa_get_update_order(eng.h, _lib.C.byref(v)))
    return "reference" if v.value == _lib.QA_ORDER_REFERENCE else "checkerboard"


class _Seeded:
    def __init__(self):
        self._seed = _random_seed()
        self._runs = 0

    def set_seed(self, seed: int) -> None:
        self._seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self._runs = 0

    def _next_seed(self, reads: int) -> int:
        s = (self._seed + self._runs) & 0xFFFFFFFFFFFFFFFF
        self._runs += reads
        return s


def _outs(n: int, reads: int, steps: int):
    # every entry is written by the run (unpacked best states, energies, traces)
    spins = np.empty((reads, n), dtype=np.int8)
    energies = np.empty(reads, dtype=np.float64)
    trace = np.empty((reads, steps), dtype=np.float64)
    o = _lib.qa_run_out(spins.ctypes.data, energies.ctypes.data, trace.ctypes.data)
    return o, spins, energies, trace


class Annealer(_Seeded):
    """``qanneal.Annealer(hamiltonian, schedule, backend)`` -- SA Metropolis (annealer.cpp:33-75)."""

    def __init__(self, hamiltonian, schedule: AnnealSchedule, backend: str = "cuda", device: Optional[int] = None):
        super().__init__()
        _check_backend(backend)
        if hamiltonian is None:
            raise ValueError("Annealer requires a backend.")
        if len(schedule.betas) == 0:
            raise ValueError("Schedule must contain at least one beta.")
        self.hamiltonian = hamiltonian
        self.schedule = schedule
        self.device = device
        self.last_stats: Optional[RunStats] = None

    def run(self, sweeps_per_beta: int, observer=None) -> AnnealResult:
        if observer is not None:
            return self._run_observed(sweeps_per_beta, observer)
        return self.run_reads(sweeps_per_beta, reads=1)[0]

    def _run_observed(self, sweeps_per_beta: int, observer) -> AnnealResult:
        """annealer.cpp:48-71: the kernel records the sweeps; the observer is
        then called in the reference's order.  Same result as ``run``."""
        from .observers import observer_stride, replay_sa
        if sweeps_per_beta <= 0:
            raise ValueError("sweeps_per_beta must be > 0.")
        eng = _lib.Engine.get(self.device)
        prob = self.hamiltonian._device_problem(eng)
        betas = np.ascontiguousarray(self.schedule.betas, dtype=np.float64)
        S, n, spb = len(betas), self.hamiltonian.size(), int(sweeps_per_beta)
        stride = observer_stride(observer)
        rps = -(-spb // stride)
        sweeps = hasattr(observer, "record_sweep")
        states = np.zeros((S, rps, n), np.int8) if sweeps else None
        energies = np.zeros((S, rps)) if sweeps else None
        step_states = np.zeros((S, n), np.int8)
        tr = _lib.qa_sa_trace(stride, _lib.ptr(states), _lib.ptr(energies), _lib.ptr(step_states), None)
        seed = self._next_seed(1)
        prm = _lib.qa_sa_params(betas.ctypes.data, S, spb, 1, seed)
        o, spins, energy, trace = _outs(n, 1, S)
        st = _lib.qa_stats()
        probs = (C.c_void_p * 1)(prob)
        _lib.check(eng.L.qa_sa_trace_run(eng.h, probs, 1, C.byref(prm), C.byref(tr), C.byref(o), C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        replay_sa(observer, betas, spb, stride, trace[0], energies, states, step_states, State)
        return AnnealResult(State._view(spins[0]), float(energy[0]), trace[0])

    def run_reads(self, sweeps_per_beta: int, reads: int, seed: Optional[int] = None) -> List[AnnealResult]:
        if sweeps_per_beta <= 0:
            raise ValueError("sweeps_per_beta must be > 0.")
        eng = _lib.Engine.get(self.device)
        prob = self.hamiltonian._device_problem(eng)
        betas = np.ascontiguousarray(self.schedule.betas, dtype=np.float64)
        seed = self._next_seed(reads) if seed is None else int(seed)
        prm = _lib.qa_sa_params(betas.ctypes.data, len(betas), int(sweeps_per_beta), int(reads), seed)
        n = self.hamiltonian.size()
        o, spins, energies, trace = _outs(n, reads, len(betas))
        st = _lib.qa_stats()
        probs = (C.c_void_p * 1)(prob)
        _lib.check(eng.L.qa_sa_run(eng.h, probs, 1, C.byref(prm), C.byref(o), C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        return [AnnealResult(State._view(spins[r]), float(energies[r]), trace[r]) for r in range(reads)]


class ReplicaAnnealer(_Seeded):
    """``qanneal.ReplicaAnnealer(hamiltonian, schedule, replicas, backend)``
    (replica_annealer.cpp:46-142): independent SA replicas in one launch
    (replica r is the SA read keyed seed + r), with the magnetisation traces
    and the global best the reference reports."""

    def __init__(self, hamiltonian, schedule: AnnealSchedule, replicas: int, backend: str = "cuda",
                 device: Optional[int] = None):
        super().__init__()
        _check_backend(backend)
        if hamiltonian is None:
            raise ValueError("ReplicaAnnealer requires a backend.")
        if len(schedule.betas) == 0:
            raise ValueError("Schedule must contain at least one beta.")
        if replicas <= 0:
            raise ValueError("replicas must be > 0.")
        self.hamiltonian = hamiltonian
        self.schedule = schedule
        self.replicas = int(replicas)
        self.device = device
        self.last_stats: Optional[RunStats] = None

    def run(self, sweeps_per_beta: int, seed: Optional[int] = None) -> MultiAnnealResult:
        if sweeps_per_beta <= 0:
            raise ValueError("sweeps_per_beta must be > 0.")
        eng = _lib.Engine.get(self.device)
        prob = self.hamiltonian._device_problem(eng)
        betas = np.ascontiguousarray(self.schedule.betas, dtype=np.float64)
        R, S, n = self.replicas, len(betas), self.hamiltonian.size()
        seed = self._next_seed(R) if seed is None else int(seed)
        prm = _lib.qa_sa_params(betas.ctypes.data, S, int(sweeps_per_beta), R, seed)
        spins = np.zeros((R, n), np.int8)
        best = np.zeros(R)
        trace = np.zeros((R, S))
        mag = np.zeros((R, S))
        bstep = np.zeros(R, np.int32)
        o = _lib.qa_replica_out(spins.ctypes.data, best.ctypes.data, trace.ctypes.data, mag.ctypes.data,
                                bstep.ctypes.data)
        st = _lib.qa_stats()
        probs = (C.c_void_p * 1)(prob)
        _lib.check(eng.L.qa_replica_run(eng.h, probs, 1, C.byref(prm), C.byref(o), C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        reps = [ReplicaResult(State._view(spins[r]), float(best[r]), trace[r], mag[r]) for r in range(R)]
        # replica_annealer.cpp:75-81, 112-117: the lowest energy, first reached (earliest step, then replica)
        g = min(range(R), key=lambda r: (best[r], int(bstep[r]), r))
        return MultiAnnealResult(reps, State._view(spins[g]), float(best[g]), trace.mean(axis=0), mag.mean(axis=0))


class ParallelTemperingAnnealer(_Seeded):
    """``qanneal.ParallelTemperingAnnealer(hamiltonian, betas, backend)``
    (parallel_tempering.cpp:36-122): one replica per beta, Metropolis sweeps
    and neighbour swaps, ``run_reads`` batching independent ladders."""

    def __init__(self, hamiltonian, betas: Sequence[float], backend: str = "cuda", device: Optional[int] = None):
        super().__init__()
        _check_backend(backend)
        if hamiltonian is None:
            raise ValueError("ParallelTemperingAnnealer requires a backend.")
        if len(betas) < 2:
            raise ValueError("Parallel tempering requires at least two betas.")
        self.hamiltonian = hamiltonian
        self.betas = [float(b) for b in betas]
        self.device = device
        self.last_stats: Optional[RunStats] = None

    def run(self, sweeps_per_step: int, steps: int, swap_interval: int = 1) -> ParallelTemperingResult:
        return self.run_reads(sweeps_per_step, steps, swap_interval, reads=1)[0]

    def run_reads(self, sweeps_per_step: int, steps: int, swap_interval: int = 1, reads: int = 1,
                  seed: Optional[int] = None) -> List[ParallelTemperingResult]:
        if sweeps_per_step <= 0:
            raise ValueError("sweeps_per_step must be > 0.")
        if steps <= 0:
            raise ValueError("steps must be > 0.")
        if swap_interval <= 0:
            raise ValueError("swap_interval must be > 0.")
        eng = _lib.Engine.get(self.device)
        prob = self.hamiltonian._device_problem(eng)
        betas = np.ascontiguousarray(self.betas, dtype=np.float64)
        R, n = len(betas), self.hamiltonian.size()
        seed = self._next_seed(reads) if seed is None else int(seed)
        prm = _lib.qa_pt_params(betas.ctypes.data, R, int(sweeps_per_step), int(steps), int(swap_interval),
                                int(reads), seed)
        best = np.zeros((reads, n), np.int8)
        bestE = np.zeros(reads)
        fin = np.zeros((reads, R, n), np.int8)
        finE = np.zeros((reads, R))
        avg = np.zeros((reads, steps))
        swp = np.zeros((reads, steps))
        o = _lib.qa_sqapt_out(best.ctypes.data, bestE.ctypes.data, fin.ctypes.data, finE.ctypes.data,
                              avg.ctypes.data, swp.ctypes.data)
        st = _lib.qa_stats()
        probs = (C.c_void_p * 1)(prob)
        _lib.check(eng.L.qa_pt_run(eng.h, probs, 1, C.byref(prm), C.byref(o), C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        return [ParallelTemperingResult([State._view(fin[r, k]) for k in range(R)], finE[r].tolist(), State._view(best[r]),
                                        float(bestE[r]), avg[r], swp[r]) for r in range(reads)]


class SQAAnnealer(_Seeded):
    """``qanneal.SQAAnnealer(hamiltonian, schedule, trotter_slices, replicas, backend)``
    (sqa_annealer.cpp:87-477): parity-phase slice sweeps and worldline sweeps."""

    def __init__(self, hamiltonian, schedule: SQASchedule, trotter_slices: int, replicas: int = 1,
                 backend: str = "cuda", device: Optional[int] = None):
        super().__init__()
        _check_backend(backend)
        if hamiltonian is None:
            raise ValueError("SQAAnnealer requires a backend.")
        if len(schedule.betas) == 0:
            raise ValueError("SQA schedule must contain betas.")
        if len(schedule.betas) != len(schedule.gammas):
            raise ValueError("SQA schedule betas/gammas length mismatch.")
        if trotter_slices <= 0:
            raise ValueError("trotter_slices must be > 0.")
        if replicas <= 0:
            raise ValueError("replicas must be > 0.")
        self.hamiltonian = hamiltonian
        self.schedule = schedule
        self.trotter_slices = int(trotter_slices)
        self.replicas = int(replicas)
        self.device = device
        self.last_stats: Optional[RunStats] = None

    def run(self, sweeps_per_beta: int, worldline_sweeps: int, cluster_sweeps: int = 0,
            continuous_time_slices: int = 0, observer=None) -> SQAResult:
        if observer is not None:
            return self._run_observed(sweeps_per_beta, worldline_sweeps, cluster_sweeps, continuous_time_slices,
                                      observer)
        return self.run_reads(sweeps_per_beta, worldline_sweeps, cluster_sweeps, continuous_time_slices, reads=1)[0]

    def _run_observed(self, spb: int, wls: int, cls: int, cts: int, observer) -> SQAResult:
        """sqa_annealer.cpp:318-473: the ring kernel records every replica's
        sweeps and step ends; the observer is then called in the reference's
        order.  Same result as ``run``."""
        from .observers import observer_stride, replay_sqa
        eng = _lib.Engine.get(self.device)
        prob = self.hamiltonian._device_problem(eng)
        betas = np.ascontiguousarray(self.schedule.betas, dtype=np.float64)
        gammas = np.ascontiguousarray(self.schedule.gammas, dtype=np.float64)
        S, n, K = len(betas), self.hamiltonian.size(), self.replicas
        P = cts if (cts > 0 and cts > self.trotter_slices) else self.trotter_slices
        stride = observer_stride(observer)
        rps = -(-int(spb) // stride) + -(-int(cls) // stride) + -(-int(wls) // stride)
        sweeps = hasattr(observer, "record_sweep")
        ring_states = np.zeros((K, S, rps, P, n), np.int8) if sweeps else None
        ring_E = np.zeros((K, S, rps, P)) if sweeps else None
        step_states = np.zeros((K, S + 1, P, n), np.int8)
        step_E = np.zeros((K, S + 1, P)) if sweeps else None
        tr = _lib.qa_sqa_trace(stride, _lib.ptr(ring_states), _lib.ptr(ring_E), _lib.ptr(step_states),
                               _lib.ptr(step_E), None)
        seed = self._next_seed(1)
        prm = _lib.qa_sqa_params(betas.ctypes.data, gammas.ctypes.data, S, self.trotter_slices, K, int(spb),
                                 int(wls), int(cls), int(cts), 1, seed)
        o, spins, energy, trace = _outs(n, 1, S)
        st = _lib.qa_stats()
        probs = (C.c_void_p * 1)(prob)
        _lib.check(eng.L.qa_sqa_trace_run(eng.h, probs, 1, C.byref(prm), C.byref(tr), C.byref(o), C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        replay_sqa(observer, betas, gammas, P, K, int(spb), int(cls), int(wls), stride, trace[0], ring_states,
                   ring_E, step_states, step_E)
        return SQAResult(State._view(spins[0]), float(energy[0]), trace[0])

    def run_reads(self, sweeps_per_beta: int, worldline_sweeps: int, cluster_sweeps: int = 0,
                  continuous_time_slices: int = 0, reads: int = 1, seed: Optional[int] = None) -> List[SQAResult]:
        eng = _lib.Engine.get(self.device)
        prob = self.hamiltonian._device_problem(eng)
        betas = np.ascontiguousarray(self.schedule.betas, dtype=np.float64)
        gammas = np.ascontiguousarray(self.schedule.gammas, dtype=np.float64)
        seed = self._next_seed(reads) if seed is None else int(seed)
        prm = _lib.qa_sqa_params(betas.ctypes.data, gammas.ctypes.data, len(betas), self.trotter_slices,
                                 self.replicas, int(sweeps_per_beta), int(worldline_sweeps), int(cluster_sweeps),
                                 int(continuous_time_slices), int(reads), seed)
        n = self.hamiltonian.size()
        o, spins, energies, trace = _outs(n, reads, len(betas))
        st = _lib.qa_stats()
        probs = (C.c_void_p * 1)(prob)
        autotune.apply(eng, self.hamiltonian.kind, n, self.trotter_slices, int(reads) * self.replicas)
        _lib.check(eng.L.qa_sqa_run(eng.h, probs, 1, C.byref(prm), C.byref(o), C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        return [SQAResult(State._view(spins[r]), float(energies[r]), trace[r]) for r in range(reads)]


def _write_opt_debug_csv(path: str, res: "SQAResult", beta_ramp_steps: int, alpha: float) -> None:
    """The per-step rows of run_optimal's diagnostic CSV (sqa_annealer.cpp:777-787,
    914-918): phase, step, J_perp, chi_B, the step delta_J = eps chi^-alpha."""
    try:
        f = open(path, "w")
    except OSError:
        import sys
        print(f"[qlatanneal_b200 SQA run_optimal] WARNING: could not open debug CSV '{path}'.", file=sys.stderr)
        return
    with f:
        f.write("phase,step_index,j_perp,chi_B,delta_j,eps_tilde,alpha,floor_hit,chi_B_online\n")
        eps = res.calibrated_eps_tilde
        for k, (j, chi) in enumerate(zip(res.j_perp_trace, res.chi_B_trace)):
            if k < beta_ramp_steps:
                f.write(f"beta_ramp,{k},{j:.8e},{chi:.8e},0,0,{alpha:.8e},0,\n")
            else:
                dj = eps * chi ** (-alpha) if chi > 0 else 0.0
                f.write(f"run,{k},{j:.8e},{chi:.8e},{dj:.8e},{eps:.8e},{alpha:.8e},,\n")


def _sqa_run_optimal_reads(self, beta: float, j_perp_start: float, j_perp_end: float, eps_tilde: float,
                           alpha: float = 15.0 / 14.0, num_steps: int = 100, sweeps_per_step: int = 20,
                           worldline_sweeps: int = 0, cluster_sweeps: int = 0, calib_probes: int = 12,
                           calib_sweeps: int = 10, beta_ramp_fraction: float = 0.3, beta_ramp_start: float = 0.1,
                           reads: int = 1, seed: Optional[int] = None) -> List["SQAResult"]:
    """Batched ``run_optimal``: read r keyed seed + r, all reads in one call."""
    eng = _lib.Engine.get(self.device)
    prob = self.hamiltonian._device_problem(eng)
    seed = self._next_seed(reads) if seed is None else int(seed)
    prm = _lib.qa_sqaopt_params(self.trotter_slices, self.replicas, float(beta), float(j_perp_start),
                                float(j_perp_end), float(eps_tilde), float(alpha), int(num_steps),
                                int(sweeps_per_step), int(worldline_sweeps), int(cluster_sweeps), int(calib_probes),
                                int(calib_sweeps), float(beta_ramp_fraction), float(beta_ramp_start), int(reads),
                                seed)
    n, S = self.hamiltonian.size(), max(int(num_steps), 1)
    spins = np.zeros((reads, n), np.int8)
    best = np.zeros(reads)
    tr, jt, ct = np.zeros((reads, S)), np.zeros((reads, S)), np.zeros((reads, S))
    sc = np.zeros((reads, 4))
    o = _lib.qa_sqaopt_out(spins.ctypes.data, best.ctypes.data, tr.ctypes.data, jt.ctypes.data, ct.ctypes.data,
                           sc.ctypes.data)
    st = _lib.qa_stats()
    probs = (C.c_void_p * 1)(prob)
    _lib.check(eng.L.qa_sqa_opt_run(eng.h, probs, 1, C.byref(prm), C.byref(o), C.byref(st)))
    self.last_stats = RunStats.from_c(st)
    return [SQAResult(State._view(spins[r]), float(best[r]), tr[r], jt[r].tolist(), ct[r].tolist(), float(sc[r, 0]),
                      float(sc[r, 1]), float(sc[r, 2]), float(sc[r, 3])) for r in range(reads)]


def _sqa_run_optimal(self, beta: float, j_perp_start: float, j_perp_end: float, eps_tilde: float,
                     alpha: float = 15.0 / 14.0, num_steps: int = 100, sweeps_per_step: int = 20,
                     worldline_sweeps: int = 0, cluster_sweeps: int = 0, calib_probes: int = 12,
                     calib_sweeps: int = 10, debug_csv_path: str = "", beta_ramp_fraction: float = 0.3,
                     beta_ramp_start: float = 0.1) -> "SQAResult":
    """``SQAAnnealer.run_optimal`` (sqa_annealer.cpp:499-952), one read."""
    res = self.run_optimal_reads(beta, j_perp_start, j_perp_end, eps_tilde, alpha, num_steps, sweeps_per_step,
                                 worldline_sweeps, cluster_sweeps, calib_probes, calib_sweeps, beta_ramp_fraction,
                                 beta_ramp_start, reads=1)[0]
    if debug_csv_path:
        n1 = 0
        if beta_ramp_fraction > 0.0:
            n1 = min(int(beta_ramp_fraction * num_steps), num_steps - 1)
        _write_opt_debug_csv(debug_csv_path, res, n1, alpha)
    return res


class SQAParallelTemperingAnnealer(_Seeded):
    """``qanneal.SQAParallelTemperingAnnealer(hamiltonian, betas, gammas, trotter_slices, backend)``
    (sqa_parallel_tempering.cpp:81-346): one Trotter ring per (beta, Gamma) rung,
    swaps of neighbouring rungs every ``swap_interval`` steps."""

    def __init__(self, hamiltonian, betas: Sequence[float], gammas: Sequence[float], trotter_slices: int,
                 backend: str = "cuda", device: Optional[int] = None):
        super().__init__()
        _check_backend(backend)
        if hamiltonian is None:
            raise ValueError("SQAParallelTemperingAnnealer requires a backend.")
        if len(betas) < 2 or len(betas) != len(gammas):
            raise ValueError("SQA parallel tempering requires >=2 beta/gamma pairs.")
        if trotter_slices <= 0:
            raise ValueError("trotter_slices must be > 0.")
        self.hamiltonian = hamiltonian
        self.betas = [float(b) for b in betas]
        self.gammas = [float(g) for g in gammas]
        self.trotter_slices = int(trotter_slices)
        self.device = device
        self.last_stats: Optional[RunStats] = None

    def run(self, sweeps_per_step: int, worldline_sweeps: int, steps: int, swap_interval: int = 1,
            cluster_sweeps: int = 0, continuous_time_slices: int = 0) -> SQAParallelTemperingResult:
        return self.run_reads(sweeps_per_step, worldline_sweeps, steps, swap_interval, cluster_sweeps,
                              continuous_time_slices, reads=1)[0]

    def run_reads(self, sweeps_per_step: int, worldline_sweeps: int, steps: int, swap_interval: int = 1,
                  cluster_sweeps: int = 0, continuous_time_slices: int = 0, reads: int = 1,
                  seed: Optional[int] = None) -> List[SQAParallelTemperingResult]:
        eng = _lib.Engine.get(self.device)
        prob = self.hamiltonian._device_problem(eng)
        betas = np.ascontiguousarray(self.betas, dtype=np.float64)
        gammas = np.ascontiguousarray(self.gammas, dtype=np.float64)
        R = len(betas)
        seed = self._next_seed(reads) if seed is None else int(seed)
        prm = _lib.qa_sqapt_params(betas.ctypes.data, gammas.ctypes.data, R, self.trotter_slices,
                                   int(sweeps_per_step), int(worldline_sweeps), int(steps), int(swap_interval),
                                   int(cluster_sweeps), int(continuous_time_slices), int(reads), seed)
        n = self.hamiltonian.size()
        steps_ = max(int(steps), 1)
        best = np.zeros((reads, n), np.int8)
        bestE = np.zeros(reads)
        fin = np.zeros((reads, R, n), np.int8)
        finE = np.zeros((reads, R))
        avg = np.zeros((reads, steps_))
        swp = np.zeros((reads, steps_))
        o = _lib.qa_sqapt_out(best.ctypes.data, bestE.ctypes.data, fin.ctypes.data, finE.ctypes.data,
                              avg.ctypes.data, swp.ctypes.data)
        st = _lib.qa_stats()
        probs = (C.c_void_p * 1)(prob)
        autotune.apply(eng, self.hamiltonian.kind, n, self.trotter_slices, int(reads) * R)
        _lib.check(eng.L.qa_sqapt_run(eng.h, probs, 1, C.byref(prm), C.byref(o), C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        return [SQAParallelTemperingResult([State._view(fin[r, k]) for k in range(R)], finE[r].tolist(), State._view(best[r]),
                                           float(bestE[r]), avg[r], swp[r])
                for r in range(reads)]

    def run_optimal(self, num_steps: int, sweeps_per_step: int, worldline_sweeps: int = 0, eps_tilde: float = 0.0,
                    alpha: float = 15.0 / 14.0, j_perp_end: float = 0.0, cluster_sweeps: int = 0,
                    swap_interval: int = 1, continuous_time_slices: int = 0, calib_probes: int = 12,
                    calib_sweeps: int = 10, debug_csv_path: str = "") -> SQAParallelTemperingResult:
        """``run_optimal`` (sqa_parallel_tempering.cpp:348-882), one read: every rung
        at one adaptive J_perp per step, from the hottest rung's coupling to
        ``j_perp_end`` (<= 0: the coldest rung's coupling)."""
        res = self.run_optimal_reads(num_steps, sweeps_per_step, worldline_sweeps, eps_tilde, alpha, j_perp_end,
                                     cluster_sweeps, swap_interval, continuous_time_slices, calib_probes,
                                     calib_sweeps, reads=1)[0]
        if debug_csv_path:
            _write_opt_debug_csv(debug_csv_path, res, 0, alpha)
        return res

    def run_optimal_reads(self, num_steps: int, sweeps_per_step: int, worldline_sweeps: int = 0,
                          eps_tilde: float = 0.0, alpha: float = 15.0 / 14.0, j_perp_end: float = 0.0,
                          cluster_sweeps: int = 0, swap_interval: int = 1, continuous_time_slices: int = 0,
                          calib_probes: int = 12, calib_sweeps: int = 10, reads: int = 1,
                          seed: Optional[int] = None) -> List[SQAParallelTemperingResult]:
        """Batched ``run_optimal``: read r keyed seed + r, all reads in one call."""
        eng = _lib.Engine.get(self.device)
        prob = self.hamiltonian._device_problem(eng)
        betas = np.ascontiguousarray(self.betas, dtype=np.float64)
        gammas = np.ascontiguousarray(self.gammas, dtype=np.float64)
        R = len(betas)
        seed = self._next_seed(reads) if seed is None else int(seed)
        prm = _lib.qa_sqaptopt_params(betas.ctypes.data, gammas.ctypes.data, R, self.trotter_slices,
                                      int(continuous_time_slices), int(sweeps_per_step), int(worldline_sweeps),
                                      int(cluster_sweeps), int(num_steps), int(swap_interval), float(eps_tilde),
                                      float(alpha), float(j_perp_end), int(calib_probes), int(calib_sweeps),
                                      int(reads), seed)
        n, S = self.hamiltonian.size(), max(int(num_steps), 1)
        best = np.zeros((reads, n), np.int8)
        bestE = np.zeros(reads)
        fin = np.zeros((reads, R, n), np.int8)
        finE = np.zeros((reads, R))
        avg, swp, jt, ct = np.zeros((reads, S)), np.zeros((reads, S)), np.zeros((reads, S)), np.zeros((reads, S))
        sc = np.zeros((reads, 4))
        pt = _lib.qa_sqapt_out(best.ctypes.data, bestE.ctypes.data, fin.ctypes.data, finE.ctypes.data,
                               avg.ctypes.data, swp.ctypes.data)
        o = _lib.qa_sqaptopt_out(pt, jt.ctypes.data, ct.ctypes.data, sc.ctypes.data)
        st = _lib.qa_stats()
        probs = (C.c_void_p * 1)(prob)
        _lib.check(eng.L.qa_sqapt_opt_run(eng.h, probs, 1, C.byref(prm), C.byref(o), C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        return [SQAParallelTemperingResult([State._view(fin[r, k]) for k in range(R)], finE[r].tolist(), State._view(best[r]),
                                           float(bestE[r]), avg[r], swp[r], jt[r].tolist(), ct[r].tolist(),
                                           float(sc[r, 0]), float(sc[r, 1]), float(sc[r, 2]), float(sc[r, 3]))
                for r in range(reads)]


class SQAChiAnnealer(_Seeded):
    """``qanneal.SQAChiAnnealer(hamiltonian, trotter_slices, replicas, backend)``
    (sqa_chi_annealer.cpp:146-438): pilot chi_B scan, chi-weighted schedule,
    production anneal through the parity-phase kernel."""

    def __init__(self, hamiltonian, trotter_slices: int, replicas: int = 1, backend: str = "cuda",
                 device: Optional[int] = None):
        super().__init__()
        _check_backend(backend)
        if hamiltonian is None:
            raise ValueError("SQAChiAnnealer requires a backend.")
        if trotter_slices <= 0:
            raise ValueError("trotter_slices must be > 0.")
        if replicas <= 0:
            raise ValueError("replicas must be > 0.")
        self.hamiltonian = hamiltonian
        self.trotter_slices = int(trotter_slices)
        self.replicas = int(replicas)
        self.device = device
        self.last_stats: Optional[RunStats] = None

    def run_chi(self, beta: float, gamma_start: float, gamma_end: float, num_steps: int = 100,
                sweeps_per_step: int = 20, scan_points: int = 16, scan_sweeps: int = 30, scan_burn: int = 10,
                chi_floor_fraction: float = 1e-6, driver_A0: float = 0.0, beta_ramp_fraction: float = 0.3,
                beta_ramp_start: float = 0.1, debug_csv_path: str = "") -> SQAChiResult:
        res = self.run_chi_reads(beta, gamma_start, gamma_end, num_steps, sweeps_per_step, scan_points, scan_sweeps,
                                 scan_burn, chi_floor_fraction, driver_A0, beta_ramp_fraction, beta_ramp_start,
                                 reads=1)[0]
        if debug_csv_path:
            _write_chi_debug_csv(debug_csv_path, res, beta, self.trotter_slices, beta_ramp_fraction)
        return res

    def run_chi_reads(self, beta: float, gamma_start: float, gamma_end: float, num_steps: int = 100,
                      sweeps_per_step: int = 20, scan_points: int = 16, scan_sweeps: int = 30, scan_burn: int = 10,
                      chi_floor_fraction: float = 1e-6, driver_A0: float = 0.0, beta_ramp_fraction: float = 0.3,
                      beta_ramp_start: float = 0.1, reads: int = 1, seed: Optional[int] = None,
                      scan_chi: Optional[np.ndarray] = None) -> List[SQAChiResult]:
        """Batched run_chi.  ``scan_chi`` ([reads][scan_points] or [scan_points])
        replaces the pilot scan with a given chi_B curve (e.g. a predicted one)."""
        eng = _lib.Engine.get(self.device)
        prob = self.hamiltonian._device_problem(eng)
        seed = self._next_seed(reads) if seed is None else int(seed)
        ov = None
        if scan_chi is not None:
            ov = np.ascontiguousarray(np.broadcast_to(np.asarray(scan_chi, np.float64), (reads, int(scan_points))))
        prm = _lib.qa_chi_params(self.trotter_slices, self.replicas, float(beta), float(gamma_start),
                                 float(gamma_end), int(num_steps), int(sweeps_per_step), int(scan_points),
                                 int(scan_sweeps), int(scan_burn), float(chi_floor_fraction), float(driver_A0),
                                 float(beta_ramp_fraction), float(beta_ramp_start), int(reads), seed,
                                 None if ov is None else ov.ctypes.data)
        n, S, Pt = self.hamiltonian.size(), max(int(num_steps), 1), max(int(scan_points), 1)
        a = {"best_spins": np.zeros((reads, n), np.int8), "best_energy": np.zeros(reads)}
        for k in ("energy_trace", "beta_schedule", "gamma_schedule", "s_schedule"):
            a[k] = np.zeros((reads, S))
        for k in ("scan_s", "scan_gamma", "scan_chi_B"):
            a[k] = np.zeros((reads, Pt))
        a["scalars"] = np.zeros((reads, 5))
        o = _lib.qa_chi_out(*[a[f].ctypes.data for f, _ in _lib.qa_chi_out._fields_])
        st = _lib.qa_stats()
        probs = (C.c_void_p * 1)(prob)
        autotune.apply(eng, self.hamiltonian.kind + "-chi", n, self.trotter_slices, int(reads) * self.replicas)
        _lib.check(eng.L.qa_chi_run(eng.h, probs, 1, C.byref(prm), C.byref(o), C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        out = []
        for r in range(reads):
            sc = a["scalars"][r]
            out.append(SQAChiResult(State(a["best_spins"][r]), float(a["best_energy"][r]),
                                    a["energy_trace"][r], a["beta_schedule"][r], a["gamma_schedule"][r],
                                    a["s_schedule"][r], a["scan_s"][r], a["scan_gamma"][r], a["scan_chi_B"][r],
                                    float(sc[0]), float(sc[1]), float(sc[2]), float(sc[3]), float(sc[4])))
        return out


def _trotter_coupling(beta: float, gamma: float, slices: int) -> float:
    import math
    x = max(beta * gamma / float(slices), 1e-12)
    return 0.5 * math.log(1.0 / math.tanh(x))


def _write_chi_debug_csv(path: str, res: SQAChiResult, beta: float, slices: int, ramp_fraction: float) -> None:
    """The per-point and per-step rows run_chi writes (sqa_chi_annealer.cpp:201-212, 277-280, 380-387)."""
    steps = len(res.s_schedule)
    n1 = min(int(ramp_fraction * steps), steps - 2) if ramp_fraction > 0.0 else 0
    try:
        f = open(path, "w")
    except OSError:
        import sys
        print(f"[qlatanneal_b200 run_chi] WARNING: could not open debug CSV '{path}'.", file=sys.stderr)
        return
    with f:
        f.write("phase,index,s,gamma,j_perp,chi_B,beta\n")
        for m, (s, g, c) in enumerate(zip(res.scan_s, res.scan_gamma, res.scan_chi_B)):
            f.write(f"scan,{m},{s:.8e},{g:.8e},{_trotter_coupling(beta, g, slices):.8e},{c:.8e},{beta:.8e}\n")
        for step, (s, g, b) in enumerate(zip(res.s_schedule, res.gamma_schedule, res.beta_schedule)):
            phase = "beta_ramp" if step < n1 else "run"
            f.write(f"{phase},{step},{s:.8e},{g:.8e},{_trotter_coupling(b, g, slices):.8e},,{b:.8e}\n")


SQAAnnealer.run_optimal = _sqa_run_optimal
SQAAnnealer.run_optimal_reads = _sqa_run_optimal_reads


class BatchRunner:
    """Several models of one kind in one launch: the batched form of
    ``Annealer.run_reads``, ``SQAAnnealer.run_reads`` and
    ``SQAParallelTemperingAnnealer.run_reads``.  Read r of every model is keyed
    seed + r, so model p's results equal its own single-model run with the same
    seed; models may differ in size.  The reference runs such instance sets one
    after another (its benchmark scripts loop over instances)."""

    def __init__(self, device: Optional[int] = None):
        self.device = device
        self.last_stats: Optional[RunStats] = None

    def _prep(self, models):
        if len(models) == 0:
            raise ValueError("at least one model is required.")
        eng = _lib.Engine.get(self.device)
        hdl = [m._device_problem(eng) for m in models]
        return eng, (C.c_void_p * len(hdl))(*hdl)

    def anneal(self, models, schedule: AnnealSchedule, sweeps_per_beta: int, reads: int = 1,
               seed: int = 0) -> List[List[AnnealResult]]:
        if sweeps_per_beta <= 0:
            raise ValueError("sweeps_per_beta must be > 0.")
        eng, probs = self._prep(models)
        betas = np.ascontiguousarray(schedule.betas, dtype=np.float64)
        prm = _lib.qa_sa_params(betas.ctypes.data, len(betas), int(sweeps_per_beta), int(reads), int(seed))
        outs = [_outs(m.size(), reads, len(betas)) for m in models]
        arr = (_lib.qa_run_out * len(models))(*[o[0] for o in outs])
        st = _lib.qa_stats()
        _lib.check(eng.L.qa_sa_run(eng.h, probs, len(models), C.byref(prm), arr, C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        return [[AnnealResult(State._view(sp[r]), float(en[r]), tr[r]) for r in range(reads)]
                for _, sp, en, tr in outs]

    def sqa(self, models, schedule: SQASchedule, trotter_slices: int, replicas: int = 1, sweeps_per_beta: int = 1,
            worldline_sweeps: int = 0, cluster_sweeps: int = 0, continuous_time_slices: int = 0, reads: int = 1,
            seed: int = 0) -> List[List[SQAResult]]:
        eng, probs = self._prep(models)
        betas = np.ascontiguousarray(schedule.betas, dtype=np.float64)
        gammas = np.ascontiguousarray(schedule.gammas, dtype=np.float64)
        prm = _lib.qa_sqa_params(betas.ctypes.data, gammas.ctypes.data, len(betas), int(trotter_slices),
                                 int(replicas), int(sweeps_per_beta), int(worldline_sweeps), int(cluster_sweeps),
                                 int(continuous_time_slices), int(reads), int(seed))
        outs = [_outs(m.size(), reads, len(betas)) for m in models]
        arr = (_lib.qa_run_out * len(models))(*[o[0] for o in outs])
        st = _lib.qa_stats()
        autotune.apply(eng, models[0].kind, max(m.size() for m in models), int(trotter_slices),
                       int(reads) * int(replicas) * len(models))
        _lib.check(eng.L.qa_sqa_run(eng.h, probs, len(models), C.byref(prm), arr, C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        return [[SQAResult(State._view(sp[r]), float(en[r]), tr[r]) for r in range(reads)]
                for _, sp, en, tr in outs]

    def sqapt(self, models, betas: Sequence[float], gammas: Sequence[float], trotter_slices: int,
              sweeps_per_step: int, worldline_sweeps: int, steps: int, swap_interval: int = 1,
              cluster_sweeps: int = 0, continuous_time_slices: int = 0, reads: int = 1,
              seed: int = 0) -> List[List[SQAParallelTemperingResult]]:
        if len(betas) < 2 or len(betas) != len(gammas):
            raise ValueError("SQA parallel tempering requires >=2 beta/gamma pairs.")
        eng, probs = self._prep(models)
        b = np.ascontiguousarray(betas, dtype=np.float64)
        g = np.ascontiguousarray(gammas, dtype=np.float64)
        R, S = len(b), max(int(steps), 1)
        prm = _lib.qa_sqapt_params(b.ctypes.data, g.ctypes.data, R, int(trotter_slices), int(sweeps_per_step),
                                   int(worldline_sweeps), int(steps), int(swap_interval), int(cluster_sweeps),
                                   int(continuous_time_slices), int(reads), int(seed))
        bufs = []
        for m in models:
            n = m.size()
            bufs.append((np.empty((reads, n), np.int8), np.empty(reads), np.empty((reads, R, n), np.int8),
                         np.empty((reads, R)), np.empty((reads, S)), np.empty((reads, S))))
        arr = (_lib.qa_sqapt_out * len(models))(*[
            _lib.qa_sqapt_out(*(x.ctypes.data for x in bf)) for bf in bufs])
        st = _lib.qa_stats()
        autotune.apply(eng, models[0].kind, max(m.size() for m in models), int(trotter_slices),
                       int(reads) * R * len(models))
        _lib.check(eng.L.qa_sqapt_run(eng.h, probs, len(models), C.byref(prm), arr, C.byref(st)))
        self.last_stats = RunStats.from_c(st)
        return [[SQAParallelTemperingResult([State._view(fin[r, k]) for k in range(R)], finE[r].tolist(),
                                            State._view(best[r]), float(bestE[r]), avg[r], swp[r])
                 for r in range(reads)] for best, bestE, fin, finE, avg, swp in bufs]
