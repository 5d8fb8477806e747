"""``solve()`` and its schedule helpers with qanneal's signatures (python/qanneal/solver.py).

With the CUDA engine every read of a ``solve()`` call runs in one batched
launch instead of the reference's serial read loop (solver.py:679); read r is
seeded exactly as there (``set_seed(seed + r)``).  Methods "sa", "sqa",
"sqapt" and "sqa_chi" run on the GPU.  "ctpimc" and schedule_type="optimal"
are outside the sweep engine and raise.
"""
from __future__ import annotations

import logging
import math
import os
from dataclasses import dataclass
from typing import Any, Iterable, List, Optional, Sequence, Tuple

import numpy as np

from .annealers import Annealer, SQAAnnealer, SQAChiAnnealer, SQAParallelTemperingAnnealer, _write_opt_debug_csv
from .models import AnnealSchedule, DenseIsing, HigherOrderIsing, QUBO, SparseIsing, SQASchedule

try:
    import networkx as nx  # type: ignore
except Exception:  # pragma: no cover
    nx = None


@dataclass
class SolveResult:
    """``qanneal.SolveResult`` (solver.py:51-60)."""
    method: str
    samples: List[np.ndarray]
    energies: List[float]
    best_sample: np.ndarray
    best_energy: float
    trace: Optional[List[float]]
    var_order: List[Any]
    return_bits: bool


def j_perp_from_beta_gamma(beta: float, gamma: float, trotter_slices: int = 32) -> float:
    """J_perp = 0.5 ln(1/tanh(beta gamma / M)) (solver.py:63-68)."""
    x = max(beta * gamma / trotter_slices, 1e-12)
    return 0.5 * math.log(1.0 / math.tanh(x))


def j_rms_from_problem(problem: Any, n: Optional[int] = None) -> Optional[float]:
    """RMS of the non-zero off-diagonal couplings, or None (solver.py:71-125)."""

    def _rms(M) -> Optional[float]:
        M = np.asarray(M, dtype=float)
        if M.ndim != 2 or M.shape[0] != M.shape[1]:
            return None
        off = M[np.triu_indices(M.shape[0], k=1)]
        nz = off[off != 0.0]
        if nz.size == 0:
            return None
        return float(math.sqrt(float(np.mean(nz * nz))))

    def _rms_list(vals) -> Optional[float]:
        vals = [v for v in vals if v != 0.0]
        return float(math.sqrt(sum(x * x for x in vals) / len(vals))) if vals else None

    try:
        if hasattr(problem, "couplings") and callable(getattr(problem, "couplings")):
            return _rms(problem.couplings())
        if isinstance(problem, np.ndarray):
            return _rms(problem)
        if nx is not None and isinstance(problem, nx.Graph):
            return _rms_list([float(d.get("weight", 0.0)) for _, _, d in problem.edges(data=True)])
        if isinstance(problem, dict):
            return _rms_list([float(v) for (i, j), v in problem.items() if i != j])
        if isinstance(problem, (list, tuple)) and problem and isinstance(problem[0], (list, tuple)):
            return _rms_list([float(e[2]) for e in problem if int(e[0]) != int(e[1])])
    except Exception:
        return None
    return None


def auto_schedule_sa(steps: int = 50, beta_start: float = 0.1, beta_end: float = 4.0) -> AnnealSchedule:
    return AnnealSchedule.linear(beta_start, beta_end, steps)


def auto_schedule_sqa(steps: int = 50, beta_start: float = 0.1, beta_end: float = 4.0, gamma_start: float = 5.0,
                      gamma_end: float = 0.01) -> SQASchedule:
    # linear beta, geometric Gamma (solver.py:176-186)
    betas = np.linspace(beta_start, beta_end, steps).tolist()
    gammas = np.geomspace(gamma_start, gamma_end, steps).tolist()
    return SQASchedule.from_vectors(betas, gammas)


def _guess_n(entries: Iterable[Tuple[int, int, float]]) -> int:
    m = -1
    for i, j, _ in entries:
        m = max(m, i, j)
    return m + 1


def _is_higher_order_keys(keys: Iterable[Any]) -> bool:
    for k in keys:
        if isinstance(k, (tuple, list, frozenset, set)):
            if len(k) != 2:
                return True
        else:
            return True
    return False


def _normalize_problem(problem: Any, n: Optional[int] = None, convert=None) -> Tuple[Any, List[Any], bool]:
    """(ising, var_order, returns_bits) for the input forms of solver.py:284-335.
    ``convert`` turns a QUBO into its Ising model (default ``QUBO.to_ising``;
    ``solve`` passes ``QUBO.to_ising_device``)."""
    if convert is None:
        convert = QUBO.to_ising
    if isinstance(problem, (DenseIsing, SparseIsing, HigherOrderIsing)):
        return problem, list(range(problem.size())), False
    if isinstance(problem, QUBO):
        return convert(problem), list(range(problem.size())), True
    if nx is not None and isinstance(problem, nx.Graph):
        nodes = list(problem.nodes())
        idx = {v: i for i, v in enumerate(nodes)}
        Q = np.zeros((len(nodes), len(nodes)))
        for v, d in problem.nodes(data=True):
            Q[idx[v], idx[v]] += float(d.get("bias", 0.0))
        for u, v, d in problem.edges(data=True):
            w = float(d.get("weight", 0.0))
            Q[idx[u], idx[v]] += w
            Q[idx[v], idx[u]] += w
        return convert(QUBO(Q)), nodes, True
    if isinstance(problem, np.ndarray):
        return convert(QUBO(problem)), list(range(problem.shape[0])), True
    if isinstance(problem, dict):
        if _is_higher_order_keys(problem.keys()):
            size = n
            if size is None:
                size = 1 + max(int(i) for k in problem for i in ((k,) if isinstance(k, int) else tuple(k)))
            return HigherOrderIsing(problem, size), list(range(size)), False
        if n is None:
            n = _guess_n([(i, j, float(v)) for (i, j), v in problem.items()])
        return convert(QUBO(problem, n)), list(range(n)), True
    if isinstance(problem, (list, tuple)) and problem and isinstance(problem[0], (list, tuple)):
        entries = [(int(e[0]), int(e[1]), float(e[2])) for e in problem]
        if n is None:
            n = _guess_n(entries)
        return convert(QUBO(entries, n)), list(range(n)), True
    raise ValueError("Unsupported problem type. Provide QUBO, DenseIsing, SparseIsing, HigherOrderIsing, "
                     "networkx graph, ndarray, dict, or entries list.")


def _mode_params(mode: str) -> Tuple[float, float, float, float, int, int]:
    # (p_start, p_end, gamma_mult, gamma_final_ratio, sa_step_base, sqa_step_base), solver.py:348-357
    m = mode.lower().strip()
    if m == "fast":
        return 0.85, 0.22, 2.0, 0.03, 30, 40
    if m == "accurate":
        return 0.90, 0.04, 4.5, 0.008, 110, 130
    if m != "balanced":
        raise ValueError("mode must be one of: fast, balanced, accurate")
    return 0.88, 0.10, 3.0, 0.015, 60, 80


def _estimate_delta_scale(ising: Any, probes: int = 256, seed: int = 1234) -> float:
    """0.75-quantile of |dE| over random single flips (solver.py:360-379)."""
    n = int(ising.size())
    if n <= 0:
        return 1.0
    rng = np.random.default_rng(seed)
    n_probes = int(max(32, min(probes, max(64, n * 4))))
    deltas: List[float] = []
    for _ in range(n_probes):
        spins = rng.choice([-1, 1], size=n).astype(int).tolist()
        flip = int(rng.integers(0, n))
        try:
            d = abs(float(ising.delta_energy(spins, flip)))
            if np.isfinite(d):
                deltas.append(d)
        except Exception:
            continue
    if not deltas:
        return 1.0
    return max(float(np.quantile(np.array(deltas, dtype=float), 0.75)), 1e-6)


def auto_schedule_sa_tuned(problem: Any, mode: str = "balanced", steps: Optional[int] = None, probes: int = 256,
                           seed: int = 1234, n: Optional[int] = None, beta_end_scale: float = 1.0) -> AnnealSchedule:
    ising, _, _ = _normalize_problem(problem, n=n)
    p_start, p_end, _, _, sa_base, _ = _mode_params(mode)
    scale = _estimate_delta_scale(ising, probes=probes, seed=seed)
    beta_start = -np.log(p_start) / scale
    beta_end = (-np.log(p_end) / scale) * max(beta_end_scale, 1e-6)
    if steps is None:
        steps = int(sa_base + 6 * np.sqrt(max(int(ising.size()), 1)))
    return AnnealSchedule.linear(float(beta_start), float(beta_end), max(int(steps), 4))


def auto_schedule_sqa_tuned(problem: Any, mode: str = "balanced", steps: Optional[int] = None, probes: int = 256,
                            seed: int = 1234, n: Optional[int] = None, beta_end_scale: float = 1.0,
                            gamma_end_scale: float = 1.0) -> SQASchedule:
    ising, _, _ = _normalize_problem(problem, n=n)
    p_start, p_end, gamma_mult, gamma_final_ratio, _, sqa_base = _mode_params(mode)
    scale = _estimate_delta_scale(ising, probes=probes, seed=seed)
    beta_start = -np.log(p_start) / scale
    beta_end = (-np.log(p_end) / scale) * max(beta_end_scale, 1e-6)
    gamma_start = max(gamma_mult * scale, 1e-3)
    gamma_end = max(gamma_start * gamma_final_ratio * max(gamma_end_scale, 1e-8), 1e-6)
    if steps is None:
        steps = int(sqa_base + 8 * np.sqrt(max(int(ising.size()), 1)))
    steps = max(int(steps), 6)
    return SQASchedule.from_vectors(np.linspace(beta_start, beta_end, steps).tolist(),
                                    np.geomspace(gamma_start, gamma_end, steps).tolist())


def auto_ladder_sqa_tuned(problem: Any, replicas: int = 8, mode: str = "balanced", probes: int = 256,
                          seed: int = 1234, n: Optional[int] = None) -> SQASchedule:
    ising, _, _ = _normalize_problem(problem, n=n)
    _, p_end, gamma_mult, _, _, _ = _mode_params(mode)
    scale = _estimate_delta_scale(ising, probes=probes, seed=seed)
    replicas = max(int(replicas), 2)
    beta_min = max(-np.log(0.75) / scale, 1e-4)
    beta_max = max(-np.log(p_end) / scale, beta_min * 1.5)
    gamma_max = max(gamma_mult * scale, 1e-3)
    gamma_min = max(gamma_max * 0.02, 1e-4)
    return SQASchedule.from_vectors(np.geomspace(beta_min, beta_max, replicas).tolist(),
                                    np.geomspace(gamma_max, gamma_min, replicas).tolist())


def optimal_j_perp_params(problem: Any, mode: str = "balanced", trotter_slices: int = 32, probes: int = 256,
                          seed: int = 1234, n: Optional[int] = None) -> Tuple[float, float, float]:
    """(beta, j_perp_start, j_perp_end) with beta = max(4 / j_rms, 1) (solver.py:128-167)."""
    ising, _, _ = _normalize_problem(problem, n=n)
    _, p_end, gamma_mult, gamma_final_ratio, _, _ = _mode_params(mode)
    scale = _estimate_delta_scale(ising, probes=probes, seed=seed)
    jrms = j_rms_from_problem(problem, n=n)
    beta_end = max(4.0 / jrms, 1.0) if jrms is not None and jrms > 0.0 else -np.log(p_end) / scale
    gamma_start = max(gamma_mult * scale, 1e-3)
    gamma_end = max(gamma_start * gamma_final_ratio, 1e-6)
    return (float(beta_end), j_perp_from_beta_gamma(float(beta_end), float(gamma_start), trotter_slices),
            j_perp_from_beta_gamma(float(beta_end), float(gamma_end), trotter_slices))


def solve(problem: Any, method: str = "sqa", reads: int = 1, sweeps_per_beta: int = 20, worldline_sweeps: int = 5,
          cluster_sweeps: int = 0, continuous_time_slices: int = 0, trotter_slices: int = 32, replicas: int = 1,
          ctpimc_qubits_per_update: int = 1, ctpimc_qubits_per_chain: int = 1, pt_steps: int = 50,
          swap_interval: int = 1, pt_betas: Optional[Sequence[float]] = None,
          pt_gammas: Optional[Sequence[float]] = None, schedule: Optional[Any] = None, seed: Optional[int] = None,
          backend: str = "cuda", progress: bool = True, logger: Optional[logging.Logger] = None,
          n: Optional[int] = None, return_bits: bool = False, schedule_type: str = "standard",
          optimal_eps_tilde: float = 0.0, optimal_alpha: float = 15.0 / 14.0, optimal_num_steps: Optional[int] = None,
          optimal_j_perp_start: Optional[float] = None, optimal_j_perp_end: Optional[float] = None,
          optimal_beta: Optional[float] = None, optimal_calib_probes: int = 12, optimal_calib_sweeps: int = 10,
          optimal_beta_ramp_fraction: float = 0.3, optimal_debug_csv: Optional[str] = None,
          chi_gamma_start: Optional[float] = None, chi_gamma_end: Optional[float] = None,
          chi_scan_points: int = 16, chi_scan_sweeps: int = 30, chi_scan_burn: int = 10,
          chi_floor_fraction: float = 1e-6, chi_driver_A0: float = 0.0,
          chi_curve: Optional[Any] = None) -> SolveResult:
    """qanneal's ``solve()`` (solver.py:455-789) with all reads in one GPU call.

    ``chi_curve`` (method "sqa_chi" only, an addition): a chi_B curve on the
    pilot's s grid -- or a callable ``f(ising) -> curve`` such as a trained
    :class:`qlatanneal_b200.learned.ChiCurveModel` -- used instead of the pilot
    scan.
    """
    method = method.lower().strip()
    schedule_type = schedule_type.lower().strip()
    if method not in ("sa", "sqa", "sqapt", "ctpimc", "sqa_chi"):
        raise ValueError("method must be 'sa', 'sqa', 'sqapt', 'ctpimc', or 'sqa_chi'")
    if schedule_type not in ("standard", "optimal"):
        raise ValueError("schedule_type must be 'standard' or 'optimal'")
    if method == "sqa_chi" and schedule_type != "standard":
        raise ValueError("method='sqa_chi' does not support schedule_type overrides; "
                         "leave schedule_type='standard' and use the chi_* parameters.")
    if method == "ctpimc":
        raise NotImplementedError("method='ctpimc' stays on qanneal's CPU path (not part of the sweep engine).")
    if logger is None:
        logger = logging.getLogger("qlatanneal_b200.solve")
    if reads <= 0:
        raise ValueError("reads must be > 0.")

    # QUBO inputs are converted on the GPU, straight into the model's device copy
    ising, var_order, is_qubo = _normalize_problem(problem, n=n, convert=lambda q: q.to_ising_device())
    if return_bits and not is_qubo:
        raise ValueError("return_bits=True requires a QUBO-type input (QUBO, ndarray, dict, entries list, or "
                         "networkx graph). DenseIsing and SparseIsing use Ising spins {-1, +1}; set "
                         "return_bits=False or convert your problem to QUBO first.")
    if schedule is None:
        if method in ("sqa", "sqa_chi"):
            schedule = auto_schedule_sqa()
        elif method == "sqapt":
            schedule = auto_ladder_sqa_tuned(ising, replicas=max(2, replicas))
        else:
            schedule = auto_schedule_sa()
    if seed is None:
        seed = int.from_bytes(os.urandom(8), "little") >> 1
    if progress and reads > 1:
        logger.info("Running %d reads in one batched GPU call...", reads)

    if schedule_type == "optimal" and method in ("sqa", "sqapt"):
        # solver.py:616-645: beta / J_perp range / step budget resolved once
        auto_beta, auto_jps, auto_jpe = optimal_j_perp_params(ising, trotter_slices=trotter_slices)
        beta = float(optimal_beta) if optimal_beta is not None else auto_beta
        jps = float(optimal_j_perp_start) if optimal_j_perp_start is not None else auto_jps
        if optimal_j_perp_end is not None:
            jpe = float(optimal_j_perp_end)
        else:
            jrms = j_rms_from_problem(problem, n=n)
            if jrms is not None and jrms > 0.0:
                jpe = max(jps, 5.0 * jrms)
                if jpe <= jps:
                    logger.warning("optimal schedule: 5*j_rms=%.4g <= j_perp_start=%.4g; the system starts past "
                                   "criticality and the adaptive schedule has little range to traverse. Consider "
                                   "a problem with larger j_rms.", 5.0 * jrms, jps)
            else:
                jpe = auto_jpe
        opt_steps = int(optimal_num_steps) if optimal_num_steps is not None else max(100, len(schedule.betas))

    if method == "sqa" and schedule_type == "optimal":
        # solver.py:686-702: run_optimal per read (read r keyed seed + r)
        ann = SQAAnnealer(ising, schedule, trotter_slices, replicas, backend=backend)
        res = ann.run_optimal_reads(beta, jps, jpe, optimal_eps_tilde, optimal_alpha, opt_steps, sweeps_per_beta,
                                    worldline_sweeps, cluster_sweeps, int(optimal_calib_probes),
                                    int(optimal_calib_sweeps), float(optimal_beta_ramp_fraction), reads=reads,
                                    seed=seed)
        traces = [r.energy_trace for r in res]
    elif method == "sqa":
        ann = SQAAnnealer(ising, schedule, trotter_slices, replicas, backend=backend)
        res = ann.run_reads(sweeps_per_beta, worldline_sweeps, cluster_sweeps, continuous_time_slices, reads=reads,
                            seed=seed)
        traces = [r.energy_trace for r in res]
    elif method == "sqapt":
        if pt_betas is not None or pt_gammas is not None:
            if pt_betas is None or pt_gammas is None:
                raise ValueError("pt_betas and pt_gammas must both be provided.")
            lb, lg = list(map(float, pt_betas)), list(map(float, pt_gammas))
        elif isinstance(schedule, SQASchedule) and len(schedule.betas) >= 2 and len(schedule.betas) == len(
                schedule.gammas):
            lb, lg = list(schedule.betas), list(schedule.gammas)
        else:
            ladder = auto_ladder_sqa_tuned(ising, replicas=max(2, replicas))
            lb, lg = ladder.betas, ladder.gammas
        ann = SQAParallelTemperingAnnealer(ising, lb, lg, trotter_slices, backend=backend)
        if schedule_type == "optimal":
            # solver.py:718-735: J_perp runs from the ladder's hottest coupling to jpe
            res = ann.run_optimal_reads(opt_steps, sweeps_per_beta, worldline_sweeps, optimal_eps_tilde,
                                        optimal_alpha, jpe, cluster_sweeps, swap_interval, continuous_time_slices,
                                        int(optimal_calib_probes), int(optimal_calib_sweeps), reads=reads, seed=seed)
        else:
            res = ann.run_reads(sweeps_per_beta, worldline_sweeps, pt_steps, swap_interval, cluster_sweeps,
                                continuous_time_slices, reads=reads, seed=seed)
        traces = [r.average_energy_trace for r in res]
    elif method == "sqa_chi":
        beta = float(optimal_beta) if optimal_beta is not None else optimal_j_perp_params(
            ising, trotter_slices=trotter_slices)[0]
        sg = list(getattr(schedule, "gammas", []) or [])
        g0 = float(chi_gamma_start) if chi_gamma_start is not None else (float(max(sg)) if sg else 5.0)
        g1 = float(chi_gamma_end) if chi_gamma_end is not None else (float(min(sg)) if sg else 0.01)
        if not (g0 > g1 > 0.0):
            raise ValueError(f"sqa_chi requires gamma_start > gamma_end > 0 (got {g0} and {g1}).")
        steps = int(optimal_num_steps) if optimal_num_steps is not None else max(100, len(sg) if sg else 100)
        if hasattr(chi_curve, "curve"):
            curve = chi_curve.curve(ising, beta=beta, gamma_start=g0, gamma_end=g1, slices=trotter_slices,
                                    points=chi_scan_points)
        else:
            curve = chi_curve(ising) if callable(chi_curve) else chi_curve
        ann = SQAChiAnnealer(ising, trotter_slices, replicas, backend=backend)
        res = ann.run_chi_reads(beta, g0, g1, steps, sweeps_per_beta, chi_scan_points, chi_scan_sweeps,
                                chi_scan_burn, chi_floor_fraction, chi_driver_A0, optimal_beta_ramp_fraction,
                                reads=reads, seed=seed, scan_chi=curve)
        traces = [r.energy_trace for r in res]
    else:
        ann = Annealer(ising, schedule, backend=backend)
        res = ann.run_reads(sweeps_per_beta, reads=reads, seed=seed)
        traces = [r.energy_trace for r in res]

    if optimal_debug_csv and schedule_type == "optimal" and method in ("sqa", "sqapt"):
        # each read of the reference rewrites the file: the last read's rows remain
        n1 = 0
        if method == "sqa" and optimal_beta_ramp_fraction > 0.0:
            n1 = min(int(optimal_beta_ramp_fraction * opt_steps), opt_steps - 1)
        _write_opt_debug_csv(optimal_debug_csv, res[-1], n1, optimal_alpha)
    samples, energies = [], []
    for r in res:
        spins = r.best_state.as_array().astype(int)
        samples.append(((spins + 1) // 2).astype(int) if (return_bits and is_qubo) else spins)
        energies.append(float(r.best_energy))
    best = int(np.argmin(energies))
    return SolveResult(method=method, samples=samples, energies=energies, best_sample=samples[best],
                       best_energy=energies[best], trace=list(traces[0]), var_order=var_order,
                       return_bits=return_bits)
