"""qa_sa_dense_run_noalloc: SA on caller-owned device buffers, no allocation.

This entry point serves callers whose GPU memory belongs to another allocator
(here: PyTorch's, which owns the input and output tensors) and who therefore
cannot have the library cudaMalloc inside the call.  Its results must equal the
allocating entry point's (qa_sa_run, reached through Annealer.run_reads) for
the same model, schedule and seed -- on two consecutive calls, since the calls
share one static scratch array.
"""
import ctypes as C

import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200 import _lib
from qlatanneal_b200.instances import dense_real, geometric_betas, sk_dense

pytestmark = pytest.mark.gpu


def _noalloc(L, device, h, J, c, betas, spb, reads, seed, torch):
    n = h.shape[0]
    dh = torch.tensor(h, dtype=torch.float64, device=f"cuda:{device}")
    dJ = torch.tensor(J, dtype=torch.float64, device=f"cuda:{device}")
    spins = torch.zeros(reads * n, dtype=torch.int8, device=f"cuda:{device}")
    energy = torch.zeros(reads, dtype=torch.float64, device=f"cuda:{device}")
    trace = torch.zeros(reads * len(betas), dtype=torch.float64, device=f"cuda:{device}")
    b = np.ascontiguousarray(betas, dtype=np.float64)
    prm = _lib.qa_sa_params(b.ctypes.data, len(b), spb, reads, seed)
    st = _lib.qa_stats()
    rc = L.qa_sa_dense_run_noalloc(device, None, n, C.c_void_p(dh.data_ptr()), C.c_void_p(dJ.data_ptr()), c,
                                   C.byref(prm), C.c_void_p(spins.data_ptr()), C.c_void_p(energy.data_ptr()),
                                   C.c_void_p(trace.data_ptr()), C.byref(st))
    _lib.check(rc)
    torch.cuda.synchronize(device)
    return (spins.cpu().numpy().reshape(reads, n), energy.cpu().numpy(),
            trace.cpu().numpy().reshape(reads, len(betas)), st)


@pytest.mark.parametrize("real", [False, True])
def test_noalloc_matches_allocating_entry_point(real):
    torch = pytest.importorskip("torch")
    L = _lib.load()
    L.qa_sa_dense_run_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                          C.POINTER(_lib.qa_sa_params), C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.POINTER(_lib.qa_stats)]
    device = torch.cuda.current_device()
    n, reads, spb, seed = 200, 12, 3, 4242
    if real:
        h, J = dense_real(n, 8)
        c = 0.75
    else:
        h, J = sk_dense(n, 8)
        h = np.random.default_rng(1).choice([-0.5, 0.0, 0.5], n)
        c = -1.0
    betas = geometric_betas(0.1, 5.0, 40)
    ref = qa.Annealer(qa.DenseIsing(h, J, c), qa.AnnealSchedule.from_betas(betas), device=device)
    want = ref.run_reads(spb, reads=reads, seed=seed)
    for call in range(2):
        spins, energy, trace, st = _noalloc(L, device, h, J, c, betas, spb, reads, seed, torch)
        for r in range(reads):
            np.testing.assert_array_equal(spins[r], want[r].best_state.as_array())
            if real:
                assert energy[r] == pytest.approx(want[r].best_energy, rel=1e-12, abs=1e-12)
                np.testing.assert_allclose(trace[r], want[r].energy_trace, rtol=1e-12, atol=1e-12)
            else:
                assert energy[r] == want[r].best_energy
                np.testing.assert_array_equal(trace[r], want[r].energy_trace)
        assert st.slice_attempts == reads * len(betas) * spb * n
        assert st.slice_accepts == ref.last_stats.slice_accepts


def test_noalloc_rejects_oversized_runs():
    torch = pytest.importorskip("torch")
    L = _lib.load()
    L.qa_sa_dense_run_noalloc.argtypes = [C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double,
                                          C.POINTER(_lib.qa_sa_params), C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.POINTER(_lib.qa_stats)]
    device = torch.cuda.current_device()
    n = 2100  # 4 n^2 bytes of float32 couplings alone exceed the 16 MiB scratch
    dh = torch.zeros(n, dtype=torch.float64, device=f"cuda:{device}")
    dJ = torch.zeros(n * n, dtype=torch.float64, device=f"cuda:{device}")
    out = torch.zeros(n, dtype=torch.float64, device=f"cuda:{device}")
    b = np.ones(3)
    prm = _lib.qa_sa_params(b.ctypes.data, 3, 1, 1, 0)
    rc = L.qa_sa_dense_run_noalloc(device, None, n, C.c_void_p(dh.data_ptr()), C.c_void_p(dJ.data_ptr()), 0.0,
                                   C.byref(prm), C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr()),
                                   C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.QA_ERR_ARG
    assert "scratch" in _lib.last_error()
