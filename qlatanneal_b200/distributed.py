"""Reads and instances over several GPUs: one process per GPU, torch.distributed.

The sweep engine's work units are independent (reads of one instance,
instances of a batch), so ranks share nothing while they anneal; the only
exchange is at the end, the analogue of qanneal's MPI helper
(mpi_replica.cpp:8-52): a MINLOC of the best energy over ranks, ties to the
lowest rank, and the winner's best state broadcast to every rank.

Read ``r`` of a run seeded ``s`` always uses the Philox key ``s + r``, so a
sharded solve returns, read for read, what one GPU returns for all reads.

The process group is the caller's (``nccl`` on GPUs, ``gloo`` on CPU);
nothing here starts or ends one.
"""
from __future__ import annotations

import heapq
from dataclasses import dataclass
from typing import Any, Callable, List, Optional, Sequence, Tuple

import numpy as np


def read_block(reads: int, rank: int, world: int) -> range:
    """Contiguous block of read indices of ``rank``: the first reads % world
    ranks take one read more."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("rank must lie in [0, world).")
    if reads < 0:
        raise ValueError("reads must be >= 0.")
    base, extra = divmod(int(reads), int(world))
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def lpt_partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Longest-processing-time-first assignment of work units to ranks:
    units in decreasing cost (ties by index) each go to the least-loaded rank
    (ties by rank).  Deterministic, so every rank computes the same plan."""
    if world <= 0:
        raise ValueError("world must be > 0.")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    heap = [(0.0, r) for r in range(world)]
    plan: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        plan[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    for p in plan:
        p.sort()
    return plan


def sweep_cost(n: int, trotter_slices: int = 1, rungs: int = 1, steps: int = 1, sweeps: int = 1,
               reads: int = 1) -> float:
    """Site attempts of a run: the cost model the partition balances."""
    return float(n) * trotter_slices * rungs * steps * sweeps * reads


def _device_for(group) -> Any:
    import torch
    import torch.distributed as dist
    backend = dist.get_backend(group)
    if backend == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def minloc_best(energy: float, spins: np.ndarray, group=None) -> Tuple[float, np.ndarray, int]:
    """(global best energy, its spins, owning rank) on every rank.

    MPI_Allreduce(MPI_DOUBLE_INT, MPI_MINLOC) + MPI_Bcast of the state
    (mpi_replica.cpp:39,49): the lowest energy wins, equal energies go to the
    lowest rank.  Spins are int8 +-1 (or 0/1 bits) of equal length on all ranks."""
    import torch
    import torch.distributed as dist
    dev = _device_for(group)
    world = dist.get_world_size(group)
    e = torch.tensor([float(energy)], dtype=torch.float64, device=dev)
    es = [torch.empty_like(e) for _ in range(world)]
    dist.all_gather(es, e, group=group)
    vals = [float(x.item()) for x in es]
    src = min(range(world), key=lambda r: (vals[r], r))
    s = torch.as_tensor(np.ascontiguousarray(spins, dtype=np.int8), device=dev).clone()
    src_global = dist.get_global_rank(group, src) if group is not None else src
    dist.broadcast(s, src=src_global, group=group)
    return vals[src], s.cpu().numpy(), src


def gather_energies(energies: Sequence[float], reads: int, group=None) -> np.ndarray:
    """Per-read energies of every rank's contiguous read block, in read order."""
    import torch
    import torch.distributed as dist
    dev = _device_for(group)
    world = dist.get_world_size(group)
    width = len(read_block(reads, 0, world))
    buf = torch.full((width,), float("nan"), dtype=torch.float64, device=dev)
    if len(energies):
        buf[:len(energies)] = torch.as_tensor(np.asarray(energies, np.float64), device=dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    out = []
    for r in range(world):
        k = len(read_block(reads, r, world))
        out.append(parts[r][:k].cpu().numpy())
    return np.concatenate(out) if out else np.zeros(0)


@dataclass
class ShardedSolveResult:
    """The rank's own solve() result plus the global outcome."""
    local: Any
    reads: range
    best_energy: float
    best_sample: np.ndarray
    best_rank: int
    energies: np.ndarray


def solve_sharded(problem: Any, reads: int, seed: int, group=None,
                  runner: Optional[Callable[..., Any]] = None, **kwargs) -> ShardedSolveResult:
    """``solve()`` with its reads split over the ranks of ``group``.

    Rank k runs reads read_block(reads, k, world) as one batched call seeded
    ``seed + first read``, so read r keeps its key seed + r.  ``runner``
    defaults to :func:`qlatanneal_b200.solve` and must accept
    (problem, reads=, seed=, **kwargs) and return an object with ``energies``
    and ``samples``."""
    import torch.distributed as dist
    if runner is None:
        from .solver import solve as runner
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    block = read_block(reads, rank, world)
    local = None
    if len(block):
        local = runner(problem, reads=len(block), seed=int(seed) + block.start, **kwargs)
        i = int(np.argmin(local.energies))
        e_loc, s_loc = float(local.energies[i]), np.asarray(local.samples[i], np.int8)
    else:
        e_loc = float("inf")
        s_loc = None
    n = _sample_len(local, group)
    if s_loc is None:
        s_loc = np.zeros(n, np.int8)
    best_e, best_s, src = minloc_best(e_loc, s_loc, group)
    energies = gather_energies([] if local is None else list(local.energies), reads, group)
    return ShardedSolveResult(local, block, best_e, best_s, src, energies)


def _sample_len(local: Any, group=None) -> int:
    import torch
    import torch.distributed as dist
    n = len(local.samples[0]) if local is not None else 0
    t = torch.tensor([n], dtype=torch.int64, device=_device_for(group))
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return int(t.item())


@dataclass
class ShardedSetResult:
    """An instance set run over the ranks of a group: the LPT plan, this
    rank's own per-instance results (``local[j]`` belongs to instance
    ``plan[rank][j]``) and, on every rank, each instance's best energy over its
    reads, the read that reached it and its best state."""
    plan: List[List[int]]
    local: List[Any]
    best_energy: np.ndarray
    best_read: np.ndarray
    best_state: List[np.ndarray]


_SET_METHODS = ("anneal", "sqa", "sqapt")


def _set_cost(method: str, n: int, kw: dict, reads: int) -> float:
    if method == "anneal":
        return sweep_cost(n, 1, 1, len(kw["schedule"].betas), kw["sweeps_per_beta"], reads)
    if method == "sqa":
        sweeps = kw.get("sweeps_per_beta", 1) + kw.get("worldline_sweeps", 0) + kw.get("cluster_sweeps", 0)
        return sweep_cost(n, kw["trotter_slices"] * kw.get("replicas", 1), 1, len(kw["schedule"].betas), sweeps,
                          reads)
    sweeps = kw["sweeps_per_step"] + kw["worldline_sweeps"] + kw.get("cluster_sweeps", 0)
    return sweep_cost(n, kw["trotter_slices"], len(kw["betas"]), kw["steps"], sweeps, reads)


def run_instances_sharded(method: str, models: Sequence[Any], reads: int, seed: int, group=None,
                          runner: Optional[Callable[..., Any]] = None, **kwargs) -> ShardedSetResult:
    """An instance set (``BatchRunner.anneal / sqa / sqapt``) spread over the
    ranks of ``group``: the instances are assigned by LPT on their site-attempt
    cost (``lpt_partition``; every rank computes the same plan), each rank runs
    its share as one batched launch with the same ``reads`` and ``seed`` (read
    r of every instance keeps the key seed + r, so every instance's results are
    those of the single-process run), and one all-gather brings every
    instance's best (energy, read, state) to every rank -- the per-instance
    form of the MINLOC exchange of mpi_replica.cpp:39,49.

    ``runner(method, models, reads=, seed=, **kwargs)`` defaults to a
    :class:`BatchRunner` on this rank's device and returns, per model, a list
    of per-read results with ``best_energy`` and ``best_state``."""
    import torch
    import torch.distributed as dist
    if method not in _SET_METHODS:
        raise ValueError(f"method must be one of {_SET_METHODS}.")
    if len(models) == 0:
        raise ValueError("at least one model is required.")
    if runner is None:
        def runner(meth, ms, reads, seed, **kw):
            from .annealers import BatchRunner
            return getattr(BatchRunner(), meth)(ms, reads=reads, seed=seed, **kw)
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    sizes = [int(m.size()) for m in models]
    plan = lpt_partition([_set_cost(method, n, kwargs, reads) for n in sizes], world)
    mine = plan[rank]
    local = runner(method, [models[i] for i in mine], reads=int(reads), seed=int(seed), **kwargs) if mine else []
    # one record per assigned instance: index, best energy, best read, best state (padded)
    n_max, width = max(sizes), max(len(p) for p in plan)
    rec = np.full((width, 3 + n_max), np.nan)
    for j, i in enumerate(mine):
        es = [float(r.best_energy) for r in local[j]]
        k = min(range(len(es)), key=lambda q: (es[q], q))
        st = local[j][k].best_state
        s = np.asarray(st.as_array() if hasattr(st, "as_array") else st, np.float64)
        rec[j, 0], rec[j, 1], rec[j, 2] = i, es[k], k
        rec[j, 3:3 + len(s)] = s
    dev = _device_for(group)
    t = torch.as_tensor(rec, device=dev)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    best_e = np.full(len(models), np.inf)
    best_r = np.full(len(models), -1, np.int64)
    best_s: List[np.ndarray] = [np.zeros(0, np.int8)] * len(models)
    for part in parts:
        for row in part.cpu().numpy():
            if np.isnan(row[0]):
                continue
            i = int(row[0])
            best_e[i], best_r[i] = row[1], int(row[2])
            best_s[i] = row[3:3 + sizes[i]].astype(np.int8)
    return ShardedSetResult(plan, local, best_e, best_r, best_s)


@dataclass
class MPIReplicaSummary:
    """``qanneal.mpi.MPIReplicaSummary`` (mpi_replica.hpp:13-20)."""
    rank: int
    size: int
    local_best_energy: float
    local_best_state: np.ndarray
    global_best_energy: float
    global_best_state: np.ndarray


def run_replica_anneal(hamiltonian: Any, schedule: Any, sweeps_per_beta: int, replicas_per_rank: int, seed: int,
                       group=None, runner: Optional[Callable[..., Any]] = None) -> MPIReplicaSummary:
    """``mpi::run_replica_anneal`` (mpi_replica.cpp:8-52) over
    torch.distributed: every rank runs a ReplicaAnnealer of
    ``replicas_per_rank`` replicas, then the global best is the MINLOC of the
    ranks' bests, broadcast from its rank.  Rank k's replicas use the read keys
    seed + k * replicas_per_rank + r, so no two replicas of the job share a
    random stream.  ``runner(hamiltonian, schedule, sweeps_per_beta,
    replicas, seed)`` defaults to the GPU ReplicaAnnealer and must return an
    object with ``global_best_energy`` and ``global_best_state``."""
    import torch.distributed as dist
    if replicas_per_rank <= 0:
        raise ValueError("replicas must be > 0.")
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if runner is None:
        def runner(h, sch, spb, reps, s):
            from .annealers import ReplicaAnnealer
            return ReplicaAnnealer(h, sch, reps).run(spb, seed=s)
    res = runner(hamiltonian, schedule, int(sweeps_per_beta), int(replicas_per_rank),
                 int(seed) + rank * int(replicas_per_rank))
    state = res.global_best_state
    local = np.asarray(state.as_array() if hasattr(state, "as_array") else state, np.int8)
    e, s, _ = minloc_best(float(res.global_best_energy), local, group)
    return MPIReplicaSummary(rank, world, float(res.global_best_energy), local, e, s)
