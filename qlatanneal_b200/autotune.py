"""Launch-shape autotuner of the sweep engine.

qanneal's loops have no launch shape; the engine's ring kernels do: warps per
ring, the dense +-1 kernel's ring-state form (int32 or int16 fields, coupling
bits in shared memory or read through L2), whole-grid or rotated launches, the
steps per rotated launch and the rings per rotated group.  Every choice leaves
the results unchanged bit for bit (the engine's random streams are keyed by
ring, slice, sweep and spin, not by launch); it moves only time.

``tune_sqa`` / ``tune_sqapt`` / ``tune_chi`` time candidate shapes on a run of
the caller's own workload (the first ``timing_steps`` steps of its schedule;
SQA-Chi in buckets of its own, kind "<model kind>-chi"), check that
every candidate's results agree with the automatic shape's, and cache the
fastest per bucket -- (model kind, n rounded up to a power of two, P, rings
rounded up to a power of two) -- in a JSON file.  ``use_cache(path)`` (or the
environment variable QA_TUNE_CACHE) makes later runs of the SQA, SQA-PT,
SQA-Chi and instance-set paths apply the cached shape of their bucket; the
runs a tuning times keep their candidate shape.

The search is coordinate-wise: warps per ring, then the ring-state form (dense
models), then rotation (off, or on with steps 25 / 50 / 100 and groups of 2 /
3 / 4 rings when the rings outnumber the SMs); each stage keeps the previous
stages' winners.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import os
import threading
from typing import Dict, List, Optional

from . import _lib

AUTO = {"warps_per_ring": 0, "field_form": -1, "rotate": -1, "rot_steps": 0, "rot_group": 0}

_lock = threading.Lock()
_cache: Optional[Dict[str, dict]] = None
_cache_path: Optional[str] = None
# while a tuning runs, the runs it times keep the candidate shape instead of
# taking their bucket's cached one
_suspend = threading.local()


def _pow2(x: int) -> int:
    return 1 << max(0, math.ceil(math.log2(max(1, int(x)))))


def bucket(kind: str, n: int, P: int, rings: int) -> str:
    return f"{kind}|n{_pow2(n)}|P{int(P)}|rings{_pow2(rings)}"


def default_cache_path() -> str:
    return os.environ.get("QA_TUNE_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "qlatanneal_b200",
                                                           "tune.json")


def _load(path: str) -> Dict[str, dict]:
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def use_cache(path: Optional[str]) -> None:
    """Apply the tuned shapes cached at ``path`` to later runs (None: stop)."""
    global _cache, _cache_path
    with _lock:
        _cache_path = path
        _cache = _load(path) if path else None


def _active() -> Optional[Dict[str, dict]]:
    global _cache, _cache_path
    if _cache is None and os.environ.get("QA_TUNE_CACHE"):
        use_cache(os.environ["QA_TUNE_CACHE"])
    return _cache


def lookup(kind: str, n: int, P: int, rings: int) -> Optional[dict]:
    c = _active()
    if not c:
        return None
    e = c.get(bucket(kind, n, P, rings))
    return dict(e["tuning"]) if e else None


def set_tuning(eng, tuning: Optional[dict]) -> None:
    """The context's launch shape (None or missing fields: automatic)."""
    t = dict(AUTO)
    if tuning:
        t.update({k: int(v) for k, v in tuning.items() if k in AUTO})
    _lib.check(eng.L.qa_set_tuning(eng.h, C.byref(_lib.qa_tuning(**t))))


def apply(eng, kind: str, n: int, P: int, rings: int) -> None:
    """Before a run: the cached shape of its bucket, else automatic."""
    if getattr(_suspend, "on", False) or _active() is None:
        return
    set_tuning(eng, lookup(kind, n, P, rings))


def _candidates_stage(stage: str, base: dict, kind: str, P: int, rings: int, sms: int) -> List[dict]:
    out = []
    if stage == "warps":
        for w in sorted({max(1, (P + 1) // 2), max(1, (P + 3) // 4), min(32, P)}):
            out.append(dict(base, warps_per_ring=w))
    elif stage == "form":
        if kind.split("-")[0] == "dense":
            out = [dict(base, field_form=f) for f in (-1, 0, 1, 2)]
    elif stage == "rotation":
        out = [dict(base, rotate=0)]
        if rings > sms:
            out += [dict(base, rotate=1, rot_steps=s, rot_group=g) for s in (25, 50, 100) for g in (2, 3, 4)]
    return out


def _signature(res) -> tuple:
    return tuple((float(r.best_energy), bytes(r.best_state.as_array().tobytes())) for r in res)


def _tune(key: str, run, kind: str, P: int, rings: int, cache_path: Optional[str], repeats: int = 2,
          device: Optional[int] = None) -> dict:
    eng = _lib.Engine.get(device)
    sms = _sm_count()

    def timed(tuning):
        set_tuning(eng, tuning)
        ms, sig = [], None
        _suspend.on = True
        try:
            for _ in range(repeats + 1):  # the first run warms the shape
                res, st = run()
                ms.append(st.total_ms)
                sig = _signature(res)
        finally:
            _suspend.on = False
        return float(sorted(ms[1:])[len(ms[1:]) // 2]), sig

    base = dict(AUTO)
    auto_ms, ref_sig = timed(base)
    best_ms, tried = auto_ms, [dict(tuning=dict(base), ms=auto_ms)]
    for stage in ("warps", "form", "rotation"):
        for cand in _candidates_stage(stage, base, kind, P, rings, sms):
            ms, sig = timed(cand)
            if sig != ref_sig:
                set_tuning(eng, None)
                raise RuntimeError(f"launch shape {cand} changed the results: the engine is wrong")
            tried.append(dict(tuning=cand, ms=ms))
            if ms < best_ms:
                best_ms, base = ms, cand
    set_tuning(eng, None)
    entry = dict(tuning=base, ms=best_ms, auto_ms=auto_ms, candidates=tried)
    if cache_path:
        with _lock:
            data = _load(cache_path)
            data[key] = entry
            os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
            tmp = cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
            os.replace(tmp, cache_path)
            if _cache_path == cache_path:
                use_cache(cache_path)
    return entry


def _sm_count() -> int:
    try:
        import torch
        return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    except Exception:
        return 148


def tune_sqa(annealer, sweeps_per_beta: int, worldline_sweeps: int, reads: int, cluster_sweeps: int = 0,
             timing_steps: int = 200, cache_path: Optional[str] = None, seed: int = 1) -> dict:
    """Tune the launch shape of ``annealer.run_reads(sweeps_per_beta,
    worldline_sweeps, cluster_sweeps, reads=reads)`` on the first
    ``timing_steps`` steps of its schedule; returns the cache entry."""
    from .annealers import SQAAnnealer
    from .models import SQASchedule
    m = annealer.hamiltonian
    sched = annealer.schedule
    T = min(len(sched.betas), int(timing_steps))
    short = SQAAnnealer(m, SQASchedule.from_vectors(list(sched.betas)[:T], list(sched.gammas)[:T]),
                        annealer.trotter_slices, annealer.replicas, device=annealer.device)

    def run():
        res = short.run_reads(sweeps_per_beta, worldline_sweeps, cluster_sweeps, reads=reads, seed=seed)
        return res, short.last_stats

    rings = reads * annealer.replicas
    key = bucket(m.kind, m.size(), annealer.trotter_slices, rings)
    return _tune(key, run, m.kind, annealer.trotter_slices, rings, cache_path, device=annealer.device)


def tune_sqapt(annealer, sweeps_per_step: int, worldline_sweeps: int, steps: int, swap_interval: int, reads: int,
               cluster_sweeps: int = 0, timing_steps: int = 20, cache_path: Optional[str] = None,
               seed: int = 1) -> dict:
    """Tune ``annealer.run_reads(...)`` of an SQA-PT ladder on its first
    ``timing_steps`` pt steps."""
    T = min(int(steps), int(timing_steps))

    def run():
        res = annealer.run_reads(sweeps_per_step, worldline_sweeps, T, swap_interval, cluster_sweeps, reads=reads,
                                 seed=seed)
        return res, annealer.last_stats

    m = annealer.hamiltonian
    rings = reads * len(annealer.betas)
    key = bucket(m.kind, m.size(), annealer.trotter_slices, rings)
    return _tune(key, run, m.kind, annealer.trotter_slices, rings, cache_path, device=annealer.device)


def tune_chi(annealer, reads: int, timing_steps: Optional[int] = None, cache_path: Optional[str] = None,
             seed: int = 1, **run_chi_kwargs) -> dict:
    """Tune the launch shape of ``annealer.run_chi_reads(reads=reads,
    **run_chi_kwargs)`` (an SQAChiAnnealer; pass ``scan_chi`` to time the
    production anneal without the pilot scan).  ``timing_steps`` shortens
    ``num_steps`` for the timing.  SQA-Chi has buckets of its own (kind
    "<model kind>-chi"): its production anneal keeps the checkerboard order."""
    kw = dict(run_chi_kwargs)
    if timing_steps is not None:
        kw["num_steps"] = min(int(kw.get("num_steps", 100)), int(timing_steps))

    def run():
        res = annealer.run_chi_reads(reads=reads, seed=seed, **kw)
        return res, annealer.last_stats

    m = annealer.hamiltonian
    kind = m.kind + "-chi"
    rings = reads * annealer.replicas
    key = bucket(kind, m.size(), annealer.trotter_slices, rings)
    return _tune(key, run, kind, annealer.trotter_slices, rings, cache_path, device=annealer.device)
