"""The reference-side C++ binding (include/qa_cuda_backend.hpp) compiled and run.

tests/cxx/backend_check.cpp builds a qanneal DenseIsing / SparseIsing (the
reference's own classes), wraps it in the CUDABackend a maintainer adds to
qanneal (backend.hpp:92-105), and runs SA, SQA and SQA-PT through the C ABI
from C++.  Its results must equal the Python path's (same engine, same keys)
bit for bit, and an argument error must reach C++ as std::invalid_argument.
"""
import os
import struct
import subprocess

import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200.instances import regular3, sk_dense

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tests", "cxx", "_build", "backend_check")


def _write_case(path, mode, h, J, edges, P, K, steps, spb, wls, reads, seed, betas, gammas):
    n = len(h)
    kind = 0 if J is not None else 1
    m = 0 if edges is None else len(edges)
    rungs = len(betas) if mode == 2 else 0
    with open(path, "wb") as f:
        f.write(struct.pack("<11i", mode, kind, n, P, K, steps, spb, wls, reads, m, rungs))
        f.write(struct.pack("<Q", seed))
        f.write(np.asarray(h, "<f8").tobytes())
        if kind == 0:
            f.write(np.asarray(J, "<f8").tobytes())
        else:
            for a, b, w in edges:
                f.write(struct.pack("<qqd", a, b, w))
        f.write(np.asarray(betas, "<f8").tobytes())
        if mode != 0:
            f.write(np.asarray(gammas, "<f8").tobytes())


def _run(tmp_path, *args):
    case, out = os.path.join(tmp_path, "case.bin"), os.path.join(tmp_path, "out.bin")
    _write_case(case, *args)
    subprocess.run([BIN, case, out], check=True, timeout=300)
    return np.fromfile(out, dtype=np.uint8).tobytes()


def test_backend_check_is_built():
    assert os.path.exists(BIN), "build it with __graft_entry__.build() (needs the reference headers)"


@pytest.mark.gpu
@pytest.mark.parametrize("sparse", [False, True])
def test_cxx_backend_sa_and_sqa_equal_python(tmp_path, sparse):
    n, reads, seed = 64, 3, 777
    if sparse:
        h, edges = regular3(n, 4)
        J, model = None, qa.SparseIsing(h, edges, n)
    else:
        h, J = sk_dense(n, 4)
        edges, model = None, qa.DenseIsing(h, J)
    # SA
    betas = np.geomspace(0.1, 3.0, 12)
    raw = _run(tmp_path, 0, h, J, edges, 1, 1, len(betas), 2, 0, reads, seed, betas, None)
    want = qa.Annealer(model, qa.AnnealSchedule.from_betas(betas)).run_reads(2, reads=reads, seed=seed)
    off = 0
    for r in range(reads):
        E = struct.unpack_from("<d", raw, off)[0]
        s = np.frombuffer(raw, np.int8, n, off + 8)
        tr = np.frombuffer(raw, "<f8", len(betas), off + 8 + n)
        off += 8 + n + 8 * len(betas)
        assert E == want[r].best_energy
        np.testing.assert_array_equal(s, want[r].best_state.as_array())
        np.testing.assert_array_equal(tr, want[r].energy_trace)
    assert struct.unpack_from("<d", raw, off)[0] == pytest.approx(model.energy(want[0].best_state.spins), abs=1e-9)
    # SQA
    P, K, steps = 8, 2, 10
    betas, gammas = np.full(steps, 2.0), np.linspace(2.5, 0.05, steps)
    raw = _run(tmp_path, 1, h, J, edges, P, K, steps, 1, 1, reads, seed, betas, gammas)
    want = qa.SQAAnnealer(model, qa.SQASchedule.from_vectors(betas, gammas), P, K).run_reads(1, 1, reads=reads,
                                                                                            seed=seed)
    off = 0
    for r in range(reads):
        E = struct.unpack_from("<d", raw, off)[0]
        s = np.frombuffer(raw, np.int8, n, off + 8)
        tr = np.frombuffer(raw, "<f8", steps, off + 8 + n)
        off += 8 + n + 8 * steps
        assert E == want[r].best_energy
        np.testing.assert_array_equal(s, want[r].best_state.as_array())
        np.testing.assert_array_equal(tr, want[r].energy_trace)


@pytest.mark.gpu
def test_cxx_backend_sqapt_equals_python(tmp_path):
    n, reads, seed, P, steps = 48, 2, 99, 6, 8
    h, J = sk_dense(n, 6)
    betas, gammas = np.geomspace(0.3, 3.0, 4), np.linspace(2.0, 0.1, 4)
    raw = _run(tmp_path, 2, h, J, None, P, 1, steps, 1, 1, reads, seed, betas, gammas)
    want = qa.SQAParallelTemperingAnnealer(qa.DenseIsing(h, J), betas, gammas, P).run_reads(
        1, 1, steps, 2, reads=reads, seed=seed)
    off = 0
    for r in range(reads):
        E = struct.unpack_from("<d", raw, off)[0]
        s = np.frombuffer(raw, np.int8, n, off + 8)
        fE = np.frombuffer(raw, "<f8", 4, off + 8 + n)
        avg = np.frombuffer(raw, "<f8", steps, off + 8 + n + 32)
        off += 8 + n + 32 + 8 * steps
        assert E == want[r].best_energy
        np.testing.assert_array_equal(s, want[r].best_state.as_array())
        np.testing.assert_array_equal(fE, want[r].final_energies)
        np.testing.assert_array_equal(avg, want[r].average_energy_trace)
