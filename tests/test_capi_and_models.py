"""CPU-only checks of the boundary and the host logic (no GPU calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import qlatanneal_b200 as qa
from qlatanneal_b200 import _lib
from qlatanneal_b200.instances import hubo_random, regular3, sk_dense

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"QA_API\s+[\w\s\*]*?\b(qa_\w+)\s*\(", txt)
    return names


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libqa_gpu.so not built")
    names = declared_symbols()
    assert len(names) >= 12
    lib = C.CDLL(_lib.LIB_PATH)
    for nm in names:
        assert hasattr(lib, nm), nm
    assert set(_lib.EXPORTED) <= set(names)
    lib.qa_version.restype = C.c_char_p
    assert b"sm_100a" in lib.qa_version()


def test_models_match_reference(ref):
    rng = np.random.default_rng(1)
    h, J = sk_dense(40, 2, h_sigma=0.2)
    d, rd = qa.DenseIsing(h, J, 0.5), ref.dense(h, J, 0.5)
    hs, e = regular3(30, 3)
    sp, rsp = qa.SparseIsing(hs, e, 30, -1.0), ref.sparse(30, hs, e, -1.0)
    terms = hubo_random(24, 4)
    hu = qa.HigherOrderIsing(terms, 24)
    rhu = ref.hubo(24, [(k if isinstance(k, tuple) else (k,), v) for k, v in terms.items()])
    T, D, c, hh = rhu.hubo_info()
    assert hu.num_terms() == T and hu.max_degree() == D and hu.constant() == c
    np.testing.assert_array_equal(hu.h(), hh)
    for _ in range(10):
        s = rng.choice([-1, 1], 40)
        assert d.energy(s) == pytest.approx(rd.energy(s.astype(np.int8)), abs=1e-9)
        assert d.delta_energy(s, 5) == pytest.approx(rd.delta_energy(s.astype(np.int8), 5), abs=1e-9)
        s = rng.choice([-1, 1], 30)
        assert sp.energy(s) == pytest.approx(rsp.energy(s.astype(np.int8)), abs=1e-9)
        s = rng.choice([-1, 1], 24)
        assert hu.energy(s) == pytest.approx(rhu.energy(s.astype(np.int8)), abs=1e-9)
        assert hu.delta_energy(s, 3) == pytest.approx(rhu.delta_energy(s.astype(np.int8), 3), abs=1e-9)


def test_qubo_to_ising_bitwise(ref):
    rng = np.random.default_rng(2)
    Q = rng.normal(size=(12, 12))
    d = qa.QUBO(Q).to_ising()
    h, J, c = ref.qubo_to_ising(Q)
    np.testing.assert_array_equal(d.fields(), h)
    np.testing.assert_array_equal(d.couplings(), J)
    assert d.constant() == c


def test_model_validation_errors():
    with pytest.raises(ValueError, match="h vector length mismatch"):
        qa.DenseIsing(np.zeros(3), np.zeros((4, 4)))
    with pytest.raises(ValueError, match="self-edge"):
        qa.SparseIsing(np.zeros(3), [(1, 1, 1.0)], 3)
    with pytest.raises(ValueError, match="out of range"):
        qa.SparseIsing(np.zeros(3), [(0, 5, 1.0)], 3)
    with pytest.raises(ValueError, match="State spins must be -1 or \\+1"):
        qa.DenseIsing(np.zeros(2), np.zeros((2, 2))).energy([1, 0])
    with pytest.raises(ValueError):
        qa.SQASchedule.from_vectors([1.0, 2.0], [1.0])
    with pytest.raises(ValueError):
        qa.AnnealSchedule.linear(0.1, 1.0, 0)
    with pytest.raises(ValueError, match="Unknown backend"):
        qa.Annealer(qa.DenseIsing(np.zeros(2), np.zeros((2, 2))), qa.AnnealSchedule([1.0]), backend="tpu")


def test_hubo_consolidation_rules():
    m = qa.HigherOrderIsing({(0, 1, 2): 0.7, (2, 1, 0): -0.3, (3, 3, 4, 4): 9.9, (1, 1): 2.0, 4: 1.5}, 5)
    assert m.constant() == 9.9 + 2.0
    assert m.terms() == [((0, 1, 2), 0.7 - 0.3)]
    assert m.h()[4] == 1.5
