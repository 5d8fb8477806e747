"""ctypes access to the checker libraries (test infrastructure only).

* ``Oracle`` wraps oracle/_build/libqa_oracle.so, the C restatement of the
  qanneal sweep engine under the replay model (oracle/qa_oracle.c).
* ``Ref`` wraps oracle/_ref/libqanneal_ref.so, qanneal's own unmodified C++
  sources compiled by oracle/Makefile with a thin C driver (oracle/ref_driver.cpp).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libqa_oracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libqanneal_ref.so")

_i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
_f8p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_f4p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")


def build_oracle() -> None:
    """Compile the checker libraries (the reference only where its tree exists)."""
    subprocess.run(["make", "-s", "-f", os.path.join(ROOT, "oracle", "Makefile")], check=True)


def _c64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class OracleModel:
    def __init__(self, lib, handle, kind, n):
        self._lib, self.h, self.kind, self.n = lib, handle, kind, n

    def __del__(self):
        try:
            self._lib.or_model_free(self.h)
        except Exception:
            pass


class Oracle:
    def __init__(self, path: str = ORACLE_SO):
        if not os.path.exists(path):
            build_oracle()
        L = C.CDLL(path)
        self.L = L
        L.or_philox.argtypes = [_u32p, _u32p, _u32p]
        L.or_set_update_order.argtypes = [C.c_int]
        L.or_get_update_order.restype = C.c_int
        L.or_sweep_order.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, _i32p]
        L.or_expf.argtypes = [C.c_float]
        L.or_expf.restype = C.c_float
        L.or_model_dense.argtypes = [C.c_int, _f8p, _f8p, C.c_double]
        L.or_model_dense.restype = C.c_void_p
        L.or_model_sparse.argtypes = [C.c_int, _f8p, C.c_int, _i64p, _i64p, _f8p, C.c_double]
        L.or_model_sparse.restype = C.c_void_p
        L.or_model_hubo.argtypes = [C.c_int, C.c_int, _i64p, _i64p, _f8p, C.c_double]
        L.or_model_hubo.restype = C.c_void_p
        L.or_model_free.argtypes = [C.c_void_p]
        L.or_model_info.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 3 + [C.POINTER(C.c_double)]
        L.or_model_hubo_terms.argtypes = [C.c_void_p, _i32p, _i32p, _f8p, _f8p]
        L.or_energy64.argtypes = [C.c_void_p, _i8p]
        L.or_energy64.restype = C.c_double
        L.or_energy_track.argtypes = [C.c_void_p, _i8p]
        L.or_energy_track.restype = C.c_double
        L.or_delta_energy64.argtypes = [C.c_void_p, _i8p, C.c_int]
        L.or_delta_energy64.restype = C.c_double
        L.or_fields_init.argtypes = [C.c_void_p, _i8p, _f4p]
        L.or_init_spins.argtypes = [_i8p, C.c_int, C.c_uint64, C.c_uint32, C.c_uint32]
        L.or_sa_run.argtypes = [C.c_void_p, _f8p, C.c_int, C.c_int, C.c_uint64, C.c_int, _i8p, C.POINTER(C.c_double),
                                _f8p, _i64p, C.c_void_p, C.c_void_p]
        L.or_sqa_opt_run.argtypes = ([C.c_void_p, C.c_int, C.c_int] + [C.c_double] * 5 + [C.c_int] * 6 +
                                     [C.c_double, C.c_double, C.c_uint64, C.c_int, _i8p, C.POINTER(C.c_double),
                                      _f8p, _f8p, _f8p, _f8p])
        L.or_pt_run.argtypes = [C.c_void_p, _f8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_int, _i8p,
                                C.POINTER(C.c_double), _f8p, _i8p, _f8p, _f8p, _i64p]
        L.or_sqa_run.argtypes = [C.c_void_p, _f8p, _f8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64,
                                 C.c_int, _i8p, C.POINTER(C.c_double), _f8p, _i64p, C.c_int]
        L.or_sqapt_run.argtypes = [C.c_void_p, _f8p, _f8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                   C.c_uint64, C.c_int, _i8p, C.POINTER(C.c_double), _f8p, _i8p, _f8p, _f8p, _i64p,
                                   C.c_int]
        L.or_sqapt_opt_run.argtypes = ([C.c_void_p, _f8p, _f8p] + [C.c_int] * 7 + [C.c_double] * 3 +
                                       [C.c_int, C.c_int, C.c_uint64, C.c_int, _i8p, C.POINTER(C.c_double), _f8p,
                                        _i8p] + [_f8p] * 5)
        L.or_trace_set.argtypes = [C.c_int] + [C.c_void_p] * 7
        L.or_flip_update.argtypes = [C.c_void_p, _i8p, _f4p, C.c_int]
        L.or_chi_schedule.argtypes = ([C.c_int, _f8p, _f8p, _f8p] + [C.c_double] * 4 + [C.c_int, C.c_int] +
                                      [C.c_double] * 3 + [_f8p] * 4)
        L.or_chi_run.argtypes = ([C.c_void_p, C.c_int, C.c_int] + [C.c_double] * 3 + [C.c_int] * 5 +
                                 [C.c_double] * 4 + [C.c_uint64, C.c_int, C.c_void_p, _i8p, C.POINTER(C.c_double)] +
                                 [_f8p] * 8)

    # ---- primitives
    def philox(self, ctr, key):
        out = np.zeros(4, np.uint32)
        self.L.or_philox(np.asarray(ctr, np.uint32), np.asarray(key, np.uint32), out)
        return out

    def set_update_order(self, order: str) -> None:
        """'reference' (qanneal's shuffled sequential sweeps) or 'checkerboard'."""
        if order not in ("reference", "checkerboard"):
            raise ValueError(order)
        self.L.or_set_update_order(1 if order == "reference" else 0)

    def update_order(self) -> str:
        return "reference" if self.L.or_get_update_order() else "checkerboard"

    def sweep_order(self, key, ring, sigma, tag, n):
        out = np.zeros(n, np.int32)
        self.L.or_sweep_order(key, ring, sigma, tag, n, out)
        return out

    def expf(self, y: float) -> float:
        return float(self.L.or_expf(C.c_float(y)))

    def init_spins(self, n, key, cell, tag=1):
        s = np.zeros(n, np.int8)
        self.L.or_init_spins(s, n, key, cell, tag)
        return s

    # ---- models
    def dense(self, h, J, c=0.0) -> OracleModel:
        h, J = _c64(h), _c64(J)
        n = h.shape[0]
        return OracleModel(self.L, self.L.or_model_dense(n, h, J.reshape(-1), c), "dense", n)

    def sparse(self, n, h, edges, c=0.0) -> OracleModel:
        e = list(edges)
        ei = np.array([x[0] for x in e], np.int64)
        ej = np.array([x[1] for x in e], np.int64)
        w = np.array([x[2] for x in e], np.float64)
        hdl = self.L.or_model_sparse(n, _c64(h), len(e), ei, ej, w, c)
        if not hdl:
            raise ValueError("invalid sparse model")
        return OracleModel(self.L, hdl, "sparse", n)

    def hubo(self, n, terms, c=0.0) -> OracleModel:
        """terms: list of (vars, coeff) raw terms, as HigherOrderIsing takes them."""
        ptr = [0]
        flat = []
        coef = []
        for vars_, cf in terms:
            flat.extend(int(v) for v in vars_)
            ptr.append(len(flat))
            coef.append(float(cf))
        hdl = self.L.or_model_hubo(n, len(coef), np.array(ptr, np.int64), np.array(flat + [0], np.int64),
                                   np.array(coef + [0.0], np.float64), c)
        if not hdl:
            raise ValueError("invalid hubo model")
        return OracleModel(self.L, hdl, "hubo", n)

    def hubo_terms(self, m: OracleModel):
        n, k, T, c = C.c_int(), C.c_int(), C.c_int(), C.c_double()
        self.L.or_model_info(m.h, C.byref(n), C.byref(k), C.byref(T), C.byref(c))
        tptr = np.zeros(T.value + 1, np.int32)
        h = np.zeros(n.value, np.float64)
        coef = np.zeros(max(T.value, 1), np.float64)
        # first fetch pointer array to size vars
        tvars = np.zeros(1 << 20, np.int32)
        self.L.or_model_hubo_terms(m.h, tptr, tvars, coef, h)
        return tptr, tvars[: tptr[-1]].copy(), coef[: T.value].copy(), h, c.value

    def energy64(self, m, s):
        return float(self.L.or_energy64(m.h, np.ascontiguousarray(s, np.int8)))

    def energy_track(self, m, s):
        return float(self.L.or_energy_track(m.h, np.ascontiguousarray(s, np.int8)))

    def delta_energy64(self, m, s, flip):
        return float(self.L.or_delta_energy64(m.h, np.ascontiguousarray(s, np.int8), flip))

    def flip_update(self, m, s, g, i):
        """Flip spin i of s in place and update the float32 fields g in place."""
        self.L.or_flip_update(m.h, s, g, i)

    def fields(self, m, s):
        g = np.zeros(m.n, np.float32)
        self.L.or_fields_init(m.h, np.ascontiguousarray(s, np.int8), g)
        return g

    # ---- runs (one read each)
    def sa_run(self, m, betas, sweeps_per_beta, seed, read=0):
        betas = _c64(betas)
        best = np.zeros(m.n, np.int8)
        E = C.c_double()
        trace = np.zeros(len(betas), np.float64)
        cnt = np.zeros(4, np.int64)
        self.L.or_sa_run(m.h, betas, len(betas), sweeps_per_beta, seed, read, best, C.byref(E), trace, cnt, None, None)
        return best, E.value, trace, cnt

    def replica_run(self, m, betas, sweeps_per_beta, seed, read=0):
        """SA read with the magnetisation trace and the step of the last best
        improvement: (best, best_E, trace, mag_trace, best_step)."""
        betas = _c64(betas)
        best = np.zeros(m.n, np.int8)
        E = C.c_double()
        trace = np.zeros(len(betas))
        mag = np.zeros(len(betas))
        bstep = C.c_int()
        cnt = np.zeros(4, np.int64)
        self.L.or_sa_run(m.h, betas, len(betas), sweeps_per_beta, seed, read, best, C.byref(E), trace, cnt,
                         mag.ctypes.data, C.addressof(bstep))
        return best, E.value, trace, mag, bstep.value

    def sqa_opt_run(self, m, P, K, beta, js, je, eps, alpha, steps, spb, wls, cls, probes, csweeps, ramp_fraction,
                    ramp_start, seed, read=0):
        best = np.zeros(m.n, np.int8)
        E = C.c_double()
        tr, jt, ct, sc = np.zeros(steps), np.zeros(steps), np.zeros(steps), np.zeros(4)
        rc = self.L.or_sqa_opt_run(m.h, P, K, beta, js, je, eps, alpha, steps, spb, wls, cls, probes, csweeps,
                                   ramp_fraction, ramp_start, seed, read, best, C.byref(E), tr, jt, ct, sc)
        if rc != 0:
            raise ValueError("run_optimal arguments rejected")
        return dict(best=best, best_energy=E.value, trace=tr, j_perp=jt, chi=ct, scalars=sc)

    def pt_run(self, m, betas, spb, steps, swap_interval, seed, read=0):
        """Classical PT read: (best, best_E, final_E[R], final_spins[R][n], avg_trace, swap_trace)."""
        betas = _c64(betas)
        R = len(betas)
        best = np.zeros(m.n, np.int8)
        E = C.c_double()
        fE, fs = np.zeros(R), np.zeros(R * m.n, np.int8)
        avg, swp = np.zeros(steps), np.zeros(steps)
        cnt = np.zeros(4, np.int64)
        self.L.or_pt_run(m.h, betas, R, spb, steps, swap_interval, seed, read, best, C.byref(E), fE, fs, avg, swp,
                         cnt)
        return best, E.value, fE, fs.reshape(R, m.n), avg, swp

    def sa_trace_run(self, m, betas, spb, stride, seed, read=0):
        """SA read with the sweep trace: (best, best_E, trace, states[steps][rps][n],
        energies[steps][rps], step_states[steps][n], magnetization[steps])."""
        S, rps = len(betas), -(-spb // stride)
        states, energies = np.zeros((S, rps, m.n), np.int8), np.zeros((S, rps))
        ends, mag = np.zeros((S, m.n), np.int8), np.zeros(S)
        p = lambda a: a.ctypes.data  # noqa: E731
        self.L.or_trace_set(stride, p(states), p(energies), None, None, p(ends), None, p(mag))
        try:
            best, E, trace, _ = self.sa_run(m, betas, spb, seed, read)
        finally:
            self.L.or_trace_set(0, None, None, None, None, None, None, None)
        return best, E, trace, states, energies, ends, mag

    def sqa_trace_run(self, m, betas, gammas, P, K, spb, wls, cls, stride, seed, read=0):
        """SQA read with the sweep trace: dict of ring_states[K][S][rps][P][n],
        ring_E[K][S][rps][P], step_states[K][S+1][P][n], step_E[K][S+1][P],
        magnetization[S] and the run's (best, best_E, trace)."""
        S = len(betas)
        rps = -(-spb // stride) + -(-cls // stride) + -(-wls // stride)
        rs, rE = np.zeros((K, S, rps, P, m.n), np.int8), np.zeros((K, S, rps, P))
        es, eE = np.zeros((K, S + 1, P, m.n), np.int8), np.zeros((K, S + 1, P))
        mag = np.zeros(S)
        p = lambda a: a.ctypes.data  # noqa: E731
        self.L.or_trace_set(stride, None, None, p(rs), p(rE), p(es), p(eE), p(mag))
        try:
            best, E, trace, _ = self.sqa_run(m, betas, gammas, P, K, spb, wls, seed, read, cls=cls)
        finally:
            self.L.or_trace_set(0, None, None, None, None, None, None, None)
        return dict(best=best, best_E=E, trace=trace, ring_states=rs, ring_E=rE, step_states=es, step_E=eE, mag=mag)

    def sqa_run(self, m, betas, gammas, P, K, spb, wls, seed, read=0, cls=0):
        betas, gammas = _c64(betas), _c64(gammas)
        best = np.zeros(m.n, np.int8)
        E = C.c_double()
        trace = np.zeros(len(betas), np.float64)
        cnt = np.zeros(4, np.int64)
        self.L.or_sqa_run(m.h, betas, gammas, len(betas), P, K, spb, wls, seed, read, best, C.byref(E), trace, cnt,
                          cls)
        return best, E.value, trace, cnt

    def chi_schedule(self, scan_s, scan_gamma, chi, beta, gamma_start, gamma_end, A0, slices, num_steps,
                     floor_fraction=1e-6, ramp_fraction=0.3, ramp_start=0.1):
        b, g, s = np.zeros(num_steps), np.zeros(num_steps), np.zeros(num_steps)
        sc = np.zeros(5)
        self.L.or_chi_schedule(len(chi), _c64(scan_s), _c64(scan_gamma), _c64(chi), beta, gamma_start, gamma_end, A0,
                               slices, num_steps, floor_fraction, ramp_fraction, ramp_start, b, g, s, sc)
        return b, g, s, sc

    def chi_run(self, m, P, K, beta, gamma_start, gamma_end, num_steps, spb, points, sweeps, burn, seed, read=0,
                floor_fraction=1e-6, A0=0.0, ramp_fraction=0.3, ramp_start=0.1, scan_chi_in=None):
        best = np.zeros(m.n, np.int8)
        E = C.c_double()
        out = {k: np.zeros(num_steps) for k in ("trace", "beta", "gamma", "s")}
        scan = {k: np.zeros(points) for k in ("s", "gamma", "chi")}
        sc = np.zeros(5)
        ov = None if scan_chi_in is None else _c64(scan_chi_in)
        self.L.or_chi_run(m.h, P, K, beta, gamma_start, gamma_end, num_steps, spb, points, sweeps, burn,
                          floor_fraction, A0, ramp_fraction, ramp_start, seed, read,
                          None if ov is None else ov.ctypes.data, best, C.byref(E), out["trace"], out["beta"],
                          out["gamma"], out["s"], scan["s"], scan["gamma"], scan["chi"], sc)
        return dict(best=best, best_energy=E.value, scalars=sc, **{"scan_" + k: v for k, v in scan.items()},
                    **out)

    def sqapt_run(self, m, betas, gammas, P, spb, wls, steps, swap_interval, seed, read=0, cls=0):
        """Returns (best, best_E, final_E[R], final_spins[R][n], avg_trace, swap_trace, counters)."""
        betas, gammas = _c64(betas), _c64(gammas)
        R = len(betas)
        best = np.zeros(m.n, np.int8)
        E = C.c_double()
        fE = np.zeros(R)
        fs = np.zeros(R * m.n, np.int8)
        avg = np.zeros(steps)
        swp = np.zeros(steps)
        cnt = np.zeros(4, np.int64)
        self.L.or_sqapt_run(m.h, betas, gammas, R, P, spb, wls, steps, swap_interval, seed, read, best, C.byref(E),
                            fE, fs, avg, swp, cnt, cls)
        return best, E.value, fE, fs.reshape(R, m.n), avg, swp, cnt

    def sqapt_opt_run(self, m, betas, gammas, P, spb, wls, cls, steps, swap_interval, eps, alpha, je, probes,
                      csweeps, seed, read=0):
        """SQA-PT run_optimal read (P = resolved slice count)."""
        betas, gammas = _c64(betas), _c64(gammas)
        R = len(betas)
        best = np.zeros(m.n, np.int8)
        E = C.c_double()
        fE, fs = np.zeros(R), np.zeros(R * m.n, np.int8)
        avg, swp, jt, ct, sc = np.zeros(steps), np.zeros(steps), np.zeros(steps), np.zeros(steps), np.zeros(4)
        rc = self.L.or_sqapt_opt_run(m.h, betas, gammas, R, P, spb, wls, cls, steps, swap_interval, eps, alpha, je,
                                     probes, csweeps, seed, read, best, C.byref(E), fE, fs, avg, swp, jt, ct, sc)
        if rc != 0:
            raise ValueError("run_optimal arguments rejected")
        return dict(best=best, best_energy=E.value, final_E=fE, final_spins=fs.reshape(R, m.n), avg=avg, swap=swp,
                    j_perp=jt, chi=ct, scalars=sc)


class Ref:
    """The unmodified qanneal classes (compiled from the reference sources)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        self.L = L
        L.ref_last_error.restype = C.c_char_p
        L.ref_dense_new.argtypes = [C.c_int, _f8p, _f8p, C.c_double]
        L.ref_dense_new.restype = C.c_void_p
        L.ref_sparse_new.argtypes = [C.c_int, _f8p, C.c_int, _i64p, _i64p, _f8p, C.c_double]
        L.ref_sparse_new.restype = C.c_void_p
        L.ref_hubo_new.argtypes = [C.c_int, C.c_int, _i64p, _i64p, _f8p, C.c_double]
        L.ref_hubo_new.restype = C.c_void_p
        L.ref_model_free.argtypes = [C.c_void_p]
        L.ref_qubo_to_ising.argtypes = [C.c_int, _f8p, _f8p, _f8p, C.POINTER(C.c_double)]
        L.ref_hubo_info.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double), _f8p]
        L.ref_energy.argtypes = [C.c_void_p, _i8p, C.c_int]
        L.ref_energy.restype = C.c_double
        L.ref_delta_energy.argtypes = [C.c_void_p, _i8p, C.c_int, C.c_int]
        L.ref_delta_energy.restype = C.c_double
        L.ref_fields.argtypes = [C.c_void_p, _i8p, C.c_int, _f8p]
        L.ref_update_fields.argtypes = [C.c_void_p, _f8p, _i8p, C.c_int, C.c_int, C.c_int]
        L.ref_sa_run.argtypes = [C.c_void_p, _f8p, C.c_int, C.c_int, C.c_uint64, _i8p, C.POINTER(C.c_double), _f8p]
        L.ref_sqa_run.argtypes = [C.c_void_p, _f8p, _f8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64,
                                  _i8p, C.POINTER(C.c_double), _f8p, C.c_int]
        L.ref_pt_run.argtypes = [C.c_void_p, _f8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, _i8p,
                                 C.POINTER(C.c_double), _f8p, _f8p, _f8p]
        L.ref_replica_run.argtypes = [C.c_void_p, _f8p, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_double),
                                      _f8p, _f8p]
        L.ref_sqa_opt_run.argtypes = ([C.c_void_p, C.c_int, C.c_int] + [C.c_double] * 5 +
                                      [C.c_int] * 6 + [C.c_double, C.c_double, C.c_uint64, C.POINTER(C.c_double),
                                                       _f8p, _f8p, _f8p, _f8p])
        L.ref_sqapt_run.argtypes = [C.c_void_p, _f8p, _f8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_uint64, _i8p, C.POINTER(C.c_double), _f8p, _f8p, _f8p, C.c_int]
        L.ref_sqapt_opt_run.argtypes = ([C.c_void_p, _f8p, _f8p] + [C.c_int] * 7 + [C.c_double] * 3 +
                                        [C.c_int, C.c_int, C.c_uint64, C.POINTER(C.c_double)] + [_f8p] * 6)
        L.ref_chi_run.argtypes = ([C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                   C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_uint64, _i8p, C.POINTER(C.c_double)] + [_f8p] * 8)
        L.ref_batch_run.argtypes = [C.c_void_p, C.c_int, _f8p, _f8p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_int, C.c_uint64, C.c_int, _f8p]

    def _check(self, hdl):
        if not hdl:
            raise ValueError(self.L.ref_last_error().decode())
        return hdl

    def dense(self, h, J, c=0.0):
        h, J = _c64(h), _c64(J)
        return RefModel(self, self._check(self.L.ref_dense_new(h.shape[0], h, J.reshape(-1), c)), h.shape[0])

    def sparse(self, n, h, edges, c=0.0):
        e = list(edges)
        ei = np.array([x[0] for x in e] or [0], np.int64)
        ej = np.array([x[1] for x in e] or [0], np.int64)
        w = np.array([x[2] for x in e] or [0.0], np.float64)
        return RefModel(self, self._check(self.L.ref_sparse_new(n, _c64(h), len(e), ei, ej, w, c)), n)

    def hubo(self, n, terms, c=0.0):
        ptr, flat, coef = [0], [], []
        for vars_, cf in terms:
            flat.extend(int(v) for v in vars_)
            ptr.append(len(flat))
            coef.append(float(cf))
        hdl = self.L.ref_hubo_new(n, len(coef), np.array(ptr, np.int64), np.array(flat + [0], np.int64),
                                  np.array(coef + [0.0], np.float64), c)
        return RefModel(self, self._check(hdl), n)

    def qubo_to_ising(self, Q):
        Q = _c64(Q)
        n = Q.shape[0]
        h = np.zeros(n)
        J = np.zeros(n * n)
        c = C.c_double()
        if self.L.ref_qubo_to_ising(n, Q.reshape(-1), h, J, C.byref(c)) != 0:
            raise ValueError(self.L.ref_last_error().decode())
        return h, J.reshape(n, n), c.value


class RefModel:
    def __init__(self, ref: Ref, hdl, n):
        self.ref, self.h, self.n = ref, hdl, n

    def __del__(self):
        try:
            self.ref.L.ref_model_free(self.h)
        except Exception:
            pass

    def energy(self, s):
        return float(self.ref.L.ref_energy(self.h, np.ascontiguousarray(s, np.int8), self.n))

    def delta_energy(self, s, flip):
        return float(self.ref.L.ref_delta_energy(self.h, np.ascontiguousarray(s, np.int8), self.n, flip))

    def fields(self, s):
        f = np.zeros(self.n)
        self.ref.L.ref_fields(self.h, np.ascontiguousarray(s, np.int8), self.n, f)
        return f

    def update_fields(self, f, new_s, flip, old):
        self.ref.L.ref_update_fields(self.h, f, np.ascontiguousarray(new_s, np.int8), self.n, flip, old)

    def hubo_info(self):
        T, D, c = C.c_int(), C.c_int(), C.c_double()
        h = np.zeros(self.n)
        if self.ref.L.ref_hubo_info(self.h, C.byref(T), C.byref(D), C.byref(c), h) != 0:
            raise ValueError("not a HUBO model")
        return T.value, D.value, c.value, h

    def sa_run(self, betas, spb, seed):
        betas = _c64(betas)
        best = np.zeros(self.n, np.int8)
        E = C.c_double()
        tr = np.zeros(len(betas))
        if self.ref.L.ref_sa_run(self.h, betas, len(betas), spb, seed, best, C.byref(E), tr) != 0:
            raise ValueError(self.ref.L.ref_last_error().decode())
        return best, E.value, tr

    def sqa_run(self, betas, gammas, P, K, spb, wls, seed, cls=0):
        betas, gammas = _c64(betas), _c64(gammas)
        best = np.zeros(self.n, np.int8)
        E = C.c_double()
        tr = np.zeros(len(betas))
        if self.ref.L.ref_sqa_run(self.h, betas, gammas, len(betas), P, K, spb, wls, seed, best, C.byref(E), tr,
                                  cls) != 0:
            raise ValueError(self.ref.L.ref_last_error().decode())
        return best, E.value, tr

    def chi_run(self, P, K, beta, gamma_start, gamma_end, num_steps, spb, points, sweeps, burn, seed,
                floor_fraction=1e-6, A0=0.0, ramp_fraction=0.3, ramp_start=0.1):
        best = np.zeros(self.n, np.int8)
        E = C.c_double()
        arr = {k: np.zeros(points) for k in ("scan_s", "scan_gamma", "scan_chi")}
        arr.update({k: np.zeros(num_steps) for k in ("beta", "gamma", "s", "trace")})
        sc = np.zeros(5)
        rc = self.ref.L.ref_chi_run(self.h, P, K, beta, gamma_start, gamma_end, num_steps, spb, points, sweeps, burn,
                                    floor_fraction, A0, ramp_fraction, ramp_start, seed, best, C.byref(E),
                                    arr["scan_s"], arr["scan_gamma"], arr["scan_chi"], arr["beta"], arr["gamma"],
                                    arr["s"], arr["trace"], sc)
        if rc != 0:
            raise ValueError(self.ref.L.ref_last_error().decode())
        return dict(best=best, best_energy=E.value, scalars=sc, **arr)

    def pt_run(self, betas, spb, steps, swap_interval, seed):
        betas = _c64(betas)
        R = len(betas)
        best = np.zeros(self.n, np.int8)
        E = C.c_double()
        fE, avg, swp = np.zeros(R), np.zeros(steps), np.zeros(steps)
        if self.ref.L.ref_pt_run(self.h, betas, R, spb, steps, swap_interval, seed, best, C.byref(E), fE, avg,
                                 swp) != 0:
            raise ValueError(self.ref.L.ref_last_error().decode())
        return best, E.value, fE, avg, swp

    def replica_run(self, betas, spb, R, seed):
        betas = _c64(betas)
        E = C.c_double()
        avg, mag = np.zeros(len(betas)), np.zeros(len(betas))
        if self.ref.L.ref_replica_run(self.h, betas, len(betas), spb, R, seed, C.byref(E), avg, mag) != 0:
            raise ValueError(self.ref.L.ref_last_error().decode())
        return E.value, avg, mag

    def sqa_opt_run(self, P, K, beta, js, je, eps, alpha, steps, spb, wls, cls, probes, csweeps, ramp_fraction,
                    ramp_start, seed):
        E = C.c_double()
        tr, jt, ct, sc = np.zeros(steps), np.zeros(steps), np.zeros(steps), np.zeros(4)
        if self.ref.L.ref_sqa_opt_run(self.h, P, K, beta, js, je, eps, alpha, steps, spb, wls, cls, probes, csweeps,
                                      ramp_fraction, ramp_start, seed, C.byref(E), tr, jt, ct, sc) != 0:
            raise ValueError(self.ref.L.ref_last_error().decode())
        return dict(best_energy=E.value, trace=tr, j_perp=jt, chi=ct, scalars=sc)

    def sqapt_run(self, betas, gammas, P, spb, wls, steps, swap_interval, seed, cls=0):
        betas, gammas = _c64(betas), _c64(gammas)
        R = len(betas)
        best = np.zeros(self.n, np.int8)
        E = C.c_double()
        fE, avg, swp = np.zeros(R), np.zeros(steps), np.zeros(steps)
        rc = self.ref.L.ref_sqapt_run(self.h, betas, gammas, R, P, spb, wls, steps, swap_interval, seed, best,
                                      C.byref(E), fE, avg, swp, cls)
        if rc != 0:
            raise ValueError(self.ref.L.ref_last_error().decode())
        return best, E.value, fE, avg, swp

    def sqapt_opt_run(self, betas, gammas, P, spb, wls, cls, steps, swap_interval, eps, alpha, je, probes, csweeps,
                      seed):
        betas, gammas = _c64(betas), _c64(gammas)
        R = len(betas)
        E = C.c_double()
        fE, avg, swp, jt, ct, sc = (np.zeros(R), np.zeros(steps), np.zeros(steps), np.zeros(steps), np.zeros(steps),
                                    np.zeros(4))
        rc = self.ref.L.ref_sqapt_opt_run(self.h, betas, gammas, R, P, spb, wls, cls, steps, swap_interval, eps, alpha,
                                          je, probes, csweeps, seed, C.byref(E), fE, avg, swp, jt, ct, sc)
        if rc != 0:
            raise ValueError(self.ref.L.ref_last_error().decode())
        return dict(best_energy=E.value, final_E=fE, avg=avg, swap=swp, j_perp=jt, chi=ct, scalars=sc)

    def batch_run(self, method, betas, gammas, steps, P, K, spb, wls, reads, seed, threads):
        out = np.zeros(reads)
        g = _c64(gammas if gammas is not None else np.zeros(steps))
        rc = self.ref.L.ref_batch_run(self.h, method, _c64(betas), g, steps, P, K, spb, wls, reads, seed, threads, out)
        if rc != 0:
            raise ValueError(self.ref.L.ref_last_error().decode())
        return out
