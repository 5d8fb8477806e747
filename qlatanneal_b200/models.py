"""Problem models with qanneal's Python-visible API (python/bindings.cpp:118-320).

These are host objects.  Their float64 ``energy`` / ``delta_energy`` follow the
reference definitions (dense_ising.cpp:29-62, sparse_ising.cpp:43-71,
higher_order_ising.cpp:92-136); the sweep engine sees them through
``_upload(engine)``, which creates the device copy once (qa_problem_*).
"""
from __future__ import annotations

import ctypes as C
from typing import Any, Dict, Iterable, List, Sequence, Tuple

import numpy as np

from . import _lib


def _spins(spins: Sequence[int], n: int) -> np.ndarray:
    s = np.asarray(list(spins) if not isinstance(spins, np.ndarray) else spins, dtype=np.int64)
    if s.ndim != 1 or s.shape[0] != n:
        raise ValueError("State size mismatch.")
    if not np.all((s == 1) | (s == -1)):
        raise ValueError("State spins must be -1 or +1.")
    return s


class State:
    """``qanneal.State``: spins in {-1, +1} (state.hpp:10-31)."""

    __slots__ = ("_spins",)

    def __init__(self, n_or_spins: Any = 0):
        if isinstance(n_or_spins, (int, np.integer)):
            self._spins = np.ones(int(n_or_spins), dtype=np.int8)
        else:
            self._spins = np.asarray(n_or_spins, dtype=np.int8).copy()

    @classmethod
    def _view(cls, spins: np.ndarray) -> "State":
        """A State over an int8 row the caller owns exclusively (no copy)."""
        st = cls.__new__(cls)
        st._spins = spins
        return st

    @property
    def spins(self) -> List[int]:
        return self._spins.astype(int).tolist()

    @spins.setter
    def spins(self, v):
        self._spins = np.asarray(v, dtype=np.int8).copy()

    def size(self) -> int:
        return int(self._spins.shape[0])

    def as_array(self) -> np.ndarray:
        return self._spins


class _DeviceModel:
    """Caches one device copy (qa_problem) per engine."""

    def _device_problem(self, engine: "_lib.Engine"):
        cache = self.__dict__.setdefault("_dev", {})
        hdl = cache.get(engine.device)
        if hdl is None:
            hdl = self._upload(engine)
            cache[engine.device] = hdl
        return hdl

    def release(self) -> None:
        """Free device copies (they are also freed when the model is collected)."""
        cache = self.__dict__.get("_dev", {})
        for dev, hdl in list(cache.items()):
            try:
                _lib.load().qa_problem_free(hdl)
            except Exception:
                pass
            cache.pop(dev, None)

    def __del__(self):
        try:
            self.release()
        except Exception:
            pass


class DenseIsing(_DeviceModel):
    """E = c + sum_i h_i s_i + sum_{i<j} J_ij s_i s_j (dense_ising.hpp:11-12)."""

    def __init__(self, h, J, c: float = 0.0):
        h = np.ascontiguousarray(h, dtype=np.float64)
        J = np.ascontiguousarray(J, dtype=np.float64)
        if h.ndim != 1:
            raise ValueError("Expected 1D array.")
        if J.ndim != 2:
            raise ValueError("Expected 2D array.")
        if J.shape[0] != J.shape[1]:
            raise ValueError("Expected square matrix.")
        n = J.shape[0]
        if h.shape[0] != n:
            raise ValueError("h vector length mismatch.")
        if n == 0:
            raise ValueError("DenseIsing size must be > 0.")
        self._h, self._Jm, self._c, self._n = h, J, float(c), n
        self._upper_cache = None

    @classmethod
    def _device_built(cls, n: int, h: np.ndarray, c: float, J_fn, device: int, handle) -> "DenseIsing":
        """A model whose device copy was built on the GPU (``handle``); the host
        coupling matrix is formed by ``J_fn`` only when something asks for it."""
        self = cls.__new__(cls)
        self._h, self._Jm, self._J_fn, self._c, self._n = h, None, J_fn, float(c), int(n)
        self._upper_cache = None
        self.__dict__["_dev"] = {device: handle}
        return self

    @property
    def _J(self) -> np.ndarray:
        if self._Jm is None:
            self._Jm = np.ascontiguousarray(self._J_fn(), dtype=np.float64)
        return self._Jm

    @property
    def _upper(self) -> np.ndarray:
        if self._upper_cache is None:
            self._upper_cache = np.triu(self._J, 1)
        return self._upper_cache

    def size(self) -> int:
        return self._n

    def couplings(self) -> np.ndarray:
        return self._J.copy()

    def fields(self) -> np.ndarray:
        return self._h.copy()

    def constant(self) -> float:
        return self._c

    def energy(self, spins) -> float:
        s = _spins(spins, self._n).astype(np.float64)
        return float(self._c + self._h @ s + s @ self._upper @ s)

    def delta_energy(self, spins, flip: int) -> float:
        s = _spins(spins, self._n).astype(np.float64)
        if not 0 <= flip < self._n:
            raise ValueError("Flip index out of range.")
        local = self._h[flip] + self._J[flip] @ s - self._J[flip, flip] * s[flip]
        return float(-2.0 * s[flip] * local)

    def _upload(self, engine):
        out = C.c_void_p()
        _lib.check(engine.L.qa_problem_dense(engine.h, self._n, _lib.ptr(self._h), _lib.ptr(self._J), self._c,
                                             C.byref(out)))
        return out

    @property
    def kind(self) -> str:
        return "dense"


class SparseEdge:
    """``qanneal.SparseEdge`` (sparse_ising.hpp:12-16)."""

    def __init__(self, i: int, j: int, value: float):
        self.i, self.j, self.value = int(i), int(j), float(value)

    def __repr__(self):
        return f"SparseEdge({self.i}, {self.j}, {self.value})"


class SparseIsing(_DeviceModel):
    """Edge-list Ising model (sparse_ising.hpp:18-59)."""

    def __init__(self, h, edges: Iterable[Any], n: int, c: float = 0.0):
        h = np.ascontiguousarray(h, dtype=np.float64)
        if h.ndim != 1:
            raise ValueError("Expected 1D array.")
        n = int(n)
        if h.shape[0] != n:
            raise ValueError("h vector length mismatch.")
        if n == 0:
            raise ValueError("SparseIsing size must be > 0.")
        ei, ej, w = [], [], []
        for e in edges:
            if isinstance(e, SparseEdge):
                a, b, v = e.i, e.j, e.value
            else:
                a, b, v = int(e[0]), int(e[1]), float(e[2])
            if a < 0 or b < 0 or a >= n or b >= n:
                raise ValueError("SparseIsing edge index out of range.")
            if a == b:
                raise ValueError("SparseIsing self-edge not allowed.")
            ei.append(a); ej.append(b); w.append(v)
        self._h, self._n, self._c = h, n, float(c)
        self._ei = np.asarray(ei, dtype=np.int64)
        self._ej = np.asarray(ej, dtype=np.int64)
        self._w = np.asarray(w, dtype=np.float64)

    def size(self) -> int:
        return self._n

    def constant(self) -> float:
        return self._c

    def edges(self) -> List[SparseEdge]:
        return [SparseEdge(a, b, v) for a, b, v in zip(self._ei, self._ej, self._w)]

    def energy(self, spins) -> float:
        s = _spins(spins, self._n).astype(np.float64)
        return float(self._c + self._h @ s + np.sum(self._w * s[self._ei] * s[self._ej]))

    def delta_energy(self, spins, flip: int) -> float:
        s = _spins(spins, self._n).astype(np.float64)
        if not 0 <= flip < self._n:
            raise ValueError("Flip index out of range.")
        local = self._h[flip]
        m1 = self._ei == flip
        m2 = self._ej == flip
        local += np.sum(self._w[m1] * s[self._ej[m1]]) + np.sum(self._w[m2] * s[self._ei[m2]])
        return float(-2.0 * s[flip] * local)

    def _upload(self, engine):
        out = C.c_void_p()
        m = int(self._w.shape[0])
        _lib.check(engine.L.qa_problem_sparse(engine.h, self._n, _lib.ptr(self._h), m, _lib.ptr(self._ei),
                                              _lib.ptr(self._ej), _lib.ptr(self._w), self._c, C.byref(out)))
        return out

    @property
    def kind(self) -> str:
        return "sparse"


class QUBO:
    """``qanneal.QUBO``: x^T Q x over bits, converted by ``to_ising`` (qubo.cpp:33-69)."""

    def __init__(self, Q_or_entries, n: int = None):
        if isinstance(Q_or_entries, np.ndarray) and n is None:
            Q = np.ascontiguousarray(Q_or_entries, dtype=np.float64)
            if Q.ndim != 2:
                raise ValueError("Expected 2D array.")
            if Q.shape[0] != Q.shape[1]:
                raise ValueError("Expected square matrix.")
            if Q.shape[0] == 0:
                raise ValueError("QUBO size must be > 0.")
            self._Q = Q.copy()
        else:
            if n is None or int(n) <= 0:
                raise ValueError("QUBO size must be > 0.")
            n = int(n)
            Q = np.zeros((n, n))
            items = Q_or_entries.items() if isinstance(Q_or_entries, dict) else (
                ((e[0], e[1]), e[2]) for e in Q_or_entries)
            for key, v in items:
                if len(key) != 2:
                    raise ValueError("QUBO dict keys must be (i, j) tuples.")
                i, j = int(key[0]), int(key[1])
                if i < 0 or j < 0 or i >= n or j >= n:
                    raise ValueError("QUBO entry index out of range.")
                Q[i, j] += float(v)
            self._Q = Q

    def size(self) -> int:
        return int(self._Q.shape[0])

    def matrix(self) -> np.ndarray:
        return self._Q.copy()

    def to_ising(self) -> DenseIsing:
        # qubo.cpp:33-69: W = (Q + Q^T)/2; h = W.1/2; J = W/2 (full matrix);
        # c = tr(W)/4 + 1^T W 1/4
        # (sequential sums via cumsum, in the reference's loop order, so the
        # converted model is identical to qanneal's bit for bit)
        Q = self._Q
        n = Q.shape[0]
        W = 0.5 * (Q + Q.T)
        h = 0.5 * np.cumsum(W, axis=1)[:, -1]
        J = 0.5 * W
        seq = np.concatenate([0.25 * np.diag(W)[:, None], 0.25 * W], axis=1).reshape(-1)
        c = float(np.cumsum(seq)[-1])
        return DenseIsing(h, J, c)

    def to_ising_device(self, device: int = None) -> DenseIsing:
        """``to_ising()`` with the conversion on the GPU (``qa_problem_qubo``): Q
        goes to the device once, W, J and h are formed there straight into the
        model's device copy, c on the host meanwhile.  The model equals
        ``to_ising()`` bit for bit; its host coupling matrix is built only if
        asked for (``couplings()``, ``energy()``)."""
        eng = _lib.Engine.get(device)
        Q = self._Q
        n = Q.shape[0]
        h = np.zeros(n, dtype=np.float64)
        c = C.c_double()
        out = C.c_void_p()
        _lib.check(eng.L.qa_problem_qubo(eng.h, n, _lib.ptr(Q), _lib.ptr(h), C.byref(c), C.byref(out)))
        return DenseIsing._device_built(n, h, c.value, lambda: 0.5 * (0.5 * (Q + Q.T)), eng.device, out)


def _consolidate(n: int, raw: Iterable[Tuple[Sequence[int], float]], c: float):
    """HigherOrderIsing constructor semantics (higher_order_ising.cpp:10-90)."""
    h = np.zeros(n, dtype=np.float64)
    merged: Dict[Tuple[int, ...], float] = {}
    for vars_, coeff in raw:
        coeff = float(coeff)
        if coeff == 0.0:
            continue
        vs = sorted(int(v) for v in vars_)
        for v in vs:
            if v < 0 or v >= n:
                raise ValueError("HigherOrderIsing term variable index out of range.")
        reduced: List[int] = []
        k = 0
        while k < len(vs):
            kk = k
            while kk < len(vs) and vs[kk] == vs[k]:
                kk += 1
            if (kk - k) & 1:
                reduced.append(vs[k])
            k = kk
        if not reduced:
            c += coeff
        elif len(reduced) == 1:
            h[reduced[0]] += coeff
        else:
            key = tuple(reduced)
            merged[key] = merged.get(key, 0.0) + coeff
    terms = [(k, v) for k, v in sorted(merged.items()) if v != 0.0]
    return h, terms, c


class HigherOrderIsing(_DeviceModel):
    """E = c + sum_i h_i s_i + sum_t J_t prod_{k in t} s_k (higher_order_ising.hpp:41-110).

    ``HigherOrderIsing(terms: dict, n=None)`` or ``HigherOrderIsing(entries, n)``
    with entries ``[((i, j, k, ...), coeff), ...]``; keys may be ints (1-body).
    """

    def __init__(self, terms, n: int = None, c: float = 0.0):
        raw: List[Tuple[List[int], float]] = []
        items = terms.items() if isinstance(terms, dict) else terms
        max_idx = -1
        for key, coeff in items:
            if isinstance(key, (int, np.integer)):
                vs = [int(key)]
            else:
                try:
                    vs = [int(v) for v in key]
                except TypeError:
                    raise ValueError("HigherOrderIsing term key must be an int or an iterable of ints.")
            for v in vs:
                if v < 0:
                    raise ValueError("HigherOrderIsing term variable index out of range.")
                max_idx = max(max_idx, v)
            raw.append((vs, float(coeff)))
        if n is None:
            if max_idx < 0:
                raise ValueError("HigherOrderIsing needs at least one term.")
            n = max_idx + 1
        n = int(n)
        if n <= 0:
            raise ValueError("HigherOrderIsing size must be > 0.")
        self._n = n
        self._h, self._terms, self._c = _consolidate(n, raw, float(c))
        self._max_degree = max([len(k) for k, _ in self._terms] + ([1] if np.any(self._h != 0.0) else [0]))
        ptr = [0]
        flat: List[int] = []
        for k, _ in self._terms:
            flat.extend(k)
            ptr.append(len(flat))
        self._tptr = np.asarray(ptr, dtype=np.int64)
        self._tvars = np.asarray(flat if flat else [0], dtype=np.int32)
        self._coef = np.asarray([v for _, v in self._terms] or [0.0], dtype=np.float64)

    def size(self) -> int:
        return self._n

    def max_degree(self) -> int:
        return int(self._max_degree)

    def num_terms(self) -> int:
        return len(self._terms)

    def constant(self) -> float:
        return self._c

    def linear_terms(self) -> List[float]:
        return self._h.tolist()

    def h(self) -> np.ndarray:
        return self._h.copy()

    def terms(self) -> List[Tuple[Tuple[int, ...], float]]:
        return list(self._terms)

    def energy(self, spins) -> float:
        s = _spins(spins, self._n)
        E = self._c + float(self._h @ s)
        for k, v in self._terms:
            E += v * float(np.prod(s[list(k)]))
        return float(E)

    def coupling_energy(self, spins) -> float:
        s = _spins(spins, self._n)
        return float(sum(v * float(np.prod(s[list(k)])) for k, v in self._terms))

    def delta_energy(self, spins, flip: int) -> float:
        s = _spins(spins, self._n)
        if not 0 <= flip < self._n:
            raise ValueError("Flip index out of range.")
        local = self._h[flip]
        for k, v in self._terms:
            if flip in k:
                local += v * float(np.prod([s[x] for x in k if x != flip]))
        return float(-2.0 * s[flip] * local)

    def _upload(self, engine):
        out = C.c_void_p()
        _lib.check(engine.L.qa_problem_hubo(engine.h, self._n, _lib.ptr(self._h), len(self._terms),
                                            _lib.ptr(self._tptr), _lib.ptr(self._tvars), _lib.ptr(self._coef),
                                            self._c, C.byref(out)))
        return out

    @property
    def kind(self) -> str:
        return "hubo"


class AnnealSchedule:
    """``qanneal.AnnealSchedule`` (schedule.hpp:9-30)."""

    def __init__(self, betas: Sequence[float] = ()):
        self.betas = [float(b) for b in betas]

    def size(self) -> int:
        return len(self.betas)

    @staticmethod
    def linear(beta_start: float, beta_end: float, steps: int) -> "AnnealSchedule":
        if steps == 0:
            raise ValueError("Schedule steps must be > 0.")
        if steps == 1:
            return AnnealSchedule([beta_end])
        step = (beta_end - beta_start) / float(steps - 1)
        return AnnealSchedule([beta_start + step * float(i) for i in range(steps)])

    @staticmethod
    def from_betas(betas: Sequence[float]) -> "AnnealSchedule":
        if len(betas) == 0:
            raise ValueError("Schedule must contain betas.")
        return AnnealSchedule(betas)


class SQASchedule:
    """``qanneal.SQASchedule`` (sqa_schedule.hpp:9-28)."""

    def __init__(self, betas: Sequence[float] = (), gammas: Sequence[float] = ()):
        self.betas = [float(b) for b in betas]
        self.gammas = [float(g) for g in gammas]

    def size(self) -> int:
        return len(self.betas)

    @staticmethod
    def from_vectors(betas: Sequence[float], gammas: Sequence[float]) -> "SQASchedule":
        if len(betas) == 0:
            raise ValueError("SQA schedule must contain betas.")
        if len(betas) != len(gammas):
            raise ValueError("SQA schedule betas/gammas length mismatch.")
        return SQASchedule(betas, gammas)


def magnetization(spins) -> float:
    s = np.asarray(list(spins), dtype=np.float64)
    return float(s.mean()) if s.size else 0.0


def overlap(a, b) -> float:
    a = np.asarray(list(a), dtype=np.float64)
    b = np.asarray(list(b), dtype=np.float64)
    if a.shape != b.shape:
        raise ValueError("Spin vectors must be same length.")
    return float((a * b).mean()) if a.size else 0.0
