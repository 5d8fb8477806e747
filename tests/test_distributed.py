"""Reads sharded over ranks (gloo, world size 2, CPU): the partition, the
MINLOC/broadcast exchange, a sharded solve equal read for read to the
unsharded one (annealing by the oracle), and a rank that fails."""
import json
import os
import socket
import sys
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from qlatanneal_b200.distributed import lpt_partition, read_block, sweep_cost  # noqa: E402


def test_read_block_covers_reads():
    for reads in (0, 1, 5, 64, 257):
        for world in (1, 2, 3, 8):
            blocks = [read_block(reads, r, world) for r in range(world)]
            flat = [i for b in blocks for i in b]
            assert flat == list(range(reads))
            sizes = [len(b) for b in blocks]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        read_block(4, 2, 2)


def test_lpt_partition():
    costs = [sweep_cost(n, 16, 32, 2000, 25, 32) for n in (4096, 512, 2048, 1024, 3000, 700, 700)]
    plan = lpt_partition(costs, 3)
    assert sorted(i for p in plan for i in p) == list(range(len(costs)))
    loads = [sum(costs[i] for i in p) for p in plan]
    assert max(loads) <= 4 / 3 * (sum(costs) / 3) + max(costs)  # Graham's LPT bound, loosely
    assert plan == lpt_partition(costs, 3)  # deterministic
    assert lpt_partition([1.0, 1.0], 2) == [[0], [1]]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir, mode):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    try:
        from qlatanneal_b200.distributed import minloc_best, solve_sharded
        if mode == "solve":
            res = solve_sharded(None, reads=7, seed=41, runner=_oracle_runner)
            with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
                json.dump({"best": res.best_energy, "spins": res.best_sample.tolist(), "src": res.best_rank,
                           "energies": res.energies.tolist(), "reads": list(res.reads)}, f)
        elif mode == "set":
            from qlatanneal_b200.distributed import run_instances_sharded
            res = run_instances_sharded("anneal", _set_models(), reads=5, seed=71, runner=_oracle_set_runner,
                                        schedule=_SetSchedule(), sweeps_per_beta=2)
            with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
                json.dump({"plan": res.plan, "best": res.best_energy.tolist(), "read": res.best_read.tolist(),
                           "states": [x.tolist() for x in res.best_state],
                           "local": [[r.best_energy for r in lst] for lst in res.local]}, f)
        elif mode == "tie":
            e, s, src = minloc_best(-3.0, np.full(5, 1 if rank == 0 else -1, np.int8))
            with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
                json.dump({"best": e, "spins": s.tolist(), "src": src}, f)
        elif mode == "replica":
            from qlatanneal_b200.distributed import run_replica_anneal
            res = run_replica_anneal(None, None, 2, 3, 61, runner=_oracle_replicas)
            with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
                json.dump({"local": res.local_best_energy, "best": res.global_best_energy,
                           "spins": res.global_best_state.tolist(), "size": res.size}, f)
        elif mode == "fail":
            if rank == 1:
                raise RuntimeError("rank 1 fails before the exchange")
            try:
                minloc_best(-1.0, np.ones(4, np.int8))
                status = "returned"
            except Exception as exc:  # the peer is gone: the collective errors out
                status = "error: " + type(exc).__name__
            with open(os.path.join(out_dir, "r0.json"), "w") as f:
                json.dump({"status": status}, f)
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


_INST = dict(n=24, seed=5)


def _instance():
    from qlatanneal_b200.instances import sk_dense
    return sk_dense(_INST["n"], _INST["seed"])


def _oracle_runner(problem, reads, seed):
    """solve() stand-in that anneals on the CPU oracle: read r uses key seed + r."""
    from oracle_lib import Oracle

    class R:
        pass

    o = Oracle()
    h, J = _instance()
    m = o.dense(h, J)
    betas = np.geomspace(0.1, 3.0, 20)
    out = R()
    out.energies, out.samples = [], []
    for r in range(reads):
        best, E, _, _ = o.sa_run(m, betas, 2, seed, read=r)
        out.energies.append(E)
        out.samples.append(best)
    return out


def _oracle_replicas(h_, sched_, spb, reps, seed):
    """ReplicaAnnealer stand-in on the CPU oracle: replica r keyed seed + r,
    global best = lowest energy, earliest step, lowest replica."""
    from oracle_lib import Oracle

    class R:
        pass

    o = Oracle()
    h, J = _instance()
    m = o.dense(h, J)
    betas = np.geomspace(0.1, 3.0, 15)
    runs = [o.replica_run(m, betas, spb, seed, r) for r in range(reps)]
    g = min(range(reps), key=lambda r: (runs[r][1], runs[r][4], r))
    out = R()
    out.global_best_energy, out.global_best_state = runs[g][1], runs[g][0]
    return out


class _SetSchedule:
    betas = np.geomspace(0.1, 3.0, 12)


class _SetModel:
    def __init__(self, n, seed):
        from qlatanneal_b200.instances import sk_dense
        self.n, (self.h, self.J) = n, sk_dense(n, seed)

    def size(self):
        return self.n


def _set_models():
    # uneven sizes, so the LPT plan is not a round robin
    return [_SetModel(n, 100 + n) for n in (40, 12, 33, 20, 28, 16, 24)]


def _oracle_set_runner(method, models, reads, seed, schedule, sweeps_per_beta):
    """BatchRunner.anneal stand-in on the CPU oracle: read r of every model
    keyed seed + r."""
    from oracle_lib import Oracle

    class Res:
        def __init__(self, E, s):
            self.best_energy, self.best_state = E, s

    o = Oracle()
    out = []
    for m in models:
        om = o.dense(m.h, m.J)
        out.append([Res(*o.sa_run(om, schedule.betas, sweeps_per_beta, seed, read=r)[1::-1]) for r in range(reads)])
    return out


def test_sharded_instance_set_equals_single_process():
    """An instance set over two ranks by LPT (mpi_replica.cpp:39,49 per
    instance): both ranks end with every instance's best energy, read and
    state, equal to one process running the whole set."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    with tempfile.TemporaryDirectory() as d:
        assert _spawn("set", d)
        r0 = json.load(open(os.path.join(d, "r0.json")))
        r1 = json.load(open(os.path.join(d, "r1.json")))
    models = _set_models()
    full = _oracle_set_runner("anneal", models, 5, 71, _SetSchedule(), 2)
    assert r0["plan"] == r1["plan"] and sorted(r0["plan"][0] + r0["plan"][1]) == list(range(len(models)))
    assert r0["plan"][0] and r0["plan"][1]
    for i, reads in enumerate(full):
        es = [r.best_energy for r in reads]
        k = min(range(len(es)), key=lambda q: (es[q], q))
        for r in (r0, r1):
            assert r["best"][i] == es[k] and r["read"][i] == k
            assert r["states"][i] == np.asarray(reads[k].best_state).tolist()
    for rk, r in enumerate((r0, r1)):  # each rank's own runs are the single-process reads
        for j, i in enumerate(r["plan"][rk]):
            assert r["local"][j] == [x.best_energy for x in full[i]]


def _spawn(mode, out_dir):
    import torch.multiprocessing as tmp
    ctx = tmp.spawn(_worker, args=(2, _free_port(), out_dir, mode), nprocs=2, join=False)
    ok = True
    try:
        while not ctx.join(timeout=120):
            pass
    except Exception:
        ok = False
    return ok


def test_sharded_solve_equals_single_process():
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    with tempfile.TemporaryDirectory() as d:
        assert _spawn("solve", d)
        r0 = json.load(open(os.path.join(d, "r0.json")))
        r1 = json.load(open(os.path.join(d, "r1.json")))
    ref = _oracle_runner(None, 7, 41)
    assert r0["reads"] == [0, 1, 2, 3] and r1["reads"] == [4, 5, 6]
    assert r0["energies"] == ref.energies and r1["energies"] == ref.energies
    i = int(np.argmin(ref.energies))
    assert r0["best"] == r1["best"] == ref.energies[i]
    assert r0["spins"] == r1["spins"] == ref.samples[i].tolist()
    assert r0["src"] == (0 if i < 4 else 1)


def test_minloc_ties_go_to_lowest_rank():
    with tempfile.TemporaryDirectory() as d:
        assert _spawn("tie", d)
        r0 = json.load(open(os.path.join(d, "r0.json")))
        r1 = json.load(open(os.path.join(d, "r1.json")))
    assert r0["src"] == r1["src"] == 0
    assert r0["spins"] == r1["spins"] == [1] * 5


def test_failed_rank_ends_the_exchange_with_an_error():
    with tempfile.TemporaryDirectory() as d:
        _spawn("fail", d)  # rank 1 exits with an exception
        r0 = json.load(open(os.path.join(d, "r0.json")))
    assert r0["status"].startswith("error")


def test_replica_anneal_over_ranks():
    """mpi::run_replica_anneal (mpi_replica.cpp:8-52): each rank's replicas,
    then the MINLOC of the ranks' bests, on every rank; equal to one process
    running all 6 replicas."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    with tempfile.TemporaryDirectory() as d:
        assert _spawn("replica", d)
        r0 = json.load(open(os.path.join(d, "r0.json")))
        r1 = json.load(open(os.path.join(d, "r1.json")))
    allr = _oracle_replicas(None, None, 2, 6, 61)
    assert r0["best"] == r1["best"] == allr.global_best_energy
    assert r0["spins"] == r1["spins"]
    assert min(r0["local"], r1["local"]) == r0["best"] and r0["size"] == 2
