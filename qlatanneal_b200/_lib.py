"""ctypes binding of libqa_gpu.so (include/qa_gpu.h).

The library is built in-tree by ``qlatanneal_b200/csrc/Makefile``.  Nothing here
falls back to a CPU path: a missing library or a missing GPU raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqa_gpu.so")

QA_OK, QA_ERR_ARG, QA_ERR_CUDA, QA_ERR_OOM, QA_ERR_TIMEOUT, QA_ERR_DRIFT, QA_ERR_UNSUPPORTED = range(7)
QA_ORDER_CHECKERBOARD, QA_ORDER_REFERENCE = 0, 1

# Every symbol include/qa_gpu.h declares (checked by the CPU test suite).
EXPORTED = [
    "qa_version", "qa_last_error", "qa_device_count", "qa_create", "qa_destroy", "qa_set_drift_check",
    "qa_set_update_order", "qa_get_update_order", "qa_probe_l2_read", "qa_set_tuning", "qa_get_tuning",
    "qa_problem_dense", "qa_problem_qubo", "qa_problem_sparse", "qa_problem_hubo", "qa_problem_free", "qa_problem_size",
    "qa_sa_run", "qa_sa_trace_run", "qa_replica_run", "qa_sqa_run", "qa_sqa_trace_run", "qa_sqa_opt_run", "qa_sqapt_run", "qa_sqapt_opt_run", "qa_pt_run",
    "qa_chi_run", "qa_chi_pilot",
    "qa_mlp_create", "qa_mlp_free", "qa_mlp_num_params", "qa_mlp_get_params", "qa_mlp_set_params",
    "qa_mlp_forward", "qa_mlp_loss_grad", "qa_mlp_train_step",
]


class qa_tuning(C.Structure):
    _fields_ = [("warps_per_ring", C.c_int), ("field_form", C.c_int), ("rotate", C.c_int), ("rot_steps", C.c_int),
                ("rot_group", C.c_int)]


class qa_run_out(C.Structure):
    _fields_ = [("best_spins", C.c_void_p), ("best_energy", C.c_void_p), ("energy_trace", C.c_void_p)]


class qa_stats(C.Structure):
    _fields_ = [("slice_attempts", C.c_int64), ("slice_accepts", C.c_int64),
                ("worldline_attempts", C.c_int64), ("worldline_accepts", C.c_int64),
                ("sweep_ms", C.c_double), ("total_ms", C.c_double), ("launches", C.c_int64),
                ("sweep_launches", C.c_int64), ("h2d_bytes", C.c_int64), ("d2h_bytes", C.c_int64),
                ("max_field_drift", C.c_double)]


class qa_sa_params(C.Structure):
    _fields_ = [("betas", C.c_void_p), ("steps", C.c_int), ("sweeps_per_beta", C.c_int), ("reads", C.c_int),
                ("seed", C.c_uint64)]


class qa_sa_trace(C.Structure):
    _fields_ = [("stride", C.c_int), ("states", C.c_void_p), ("energies", C.c_void_p),
                ("step_states", C.c_void_p), ("magnetization", C.c_void_p)]


class qa_sqa_trace(C.Structure):
    _fields_ = [("stride", C.c_int), ("ring_states", C.c_void_p), ("ring_energies", C.c_void_p),
                ("step_states", C.c_void_p), ("step_energies", C.c_void_p), ("magnetization", C.c_void_p)]


class qa_replica_out(C.Structure):
    _fields_ = [("best_spins", C.c_void_p), ("best_energy", C.c_void_p), ("energy_trace", C.c_void_p),
                ("magnetization_trace", C.c_void_p), ("best_step", C.c_void_p)]


class qa_pt_params(C.Structure):
    _fields_ = [("betas", C.c_void_p), ("rungs", C.c_int), ("sweeps_per_step", C.c_int), ("steps", C.c_int),
                ("swap_interval", C.c_int), ("reads", C.c_int), ("seed", C.c_uint64)]


class qa_sqa_params(C.Structure):
    _fields_ = [("betas", C.c_void_p), ("gammas", C.c_void_p), ("steps", C.c_int), ("trotter_slices", C.c_int),
                ("replicas", C.c_int), ("sweeps_per_beta", C.c_int), ("worldline_sweeps", C.c_int),
                ("cluster_sweeps", C.c_int), ("continuous_time_slices", C.c_int), ("reads", C.c_int),
                ("seed", C.c_uint64)]


class qa_sqaopt_params(C.Structure):
    _fields_ = [("trotter_slices", C.c_int), ("replicas", C.c_int), ("beta", C.c_double),
                ("j_perp_start", C.c_double), ("j_perp_end", C.c_double), ("eps_tilde", C.c_double),
                ("alpha", C.c_double), ("num_steps", C.c_int), ("sweeps_per_step", C.c_int),
                ("worldline_sweeps", C.c_int), ("cluster_sweeps", C.c_int), ("calib_probes", C.c_int),
                ("calib_sweeps", C.c_int), ("beta_ramp_fraction", C.c_double), ("beta_ramp_start", C.c_double),
                ("reads", C.c_int), ("seed", C.c_uint64)]


class qa_sqaopt_out(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("best_spins", "best_energy", "energy_trace", "j_perp_trace",
                                         "chi_B_trace", "scalars")]


class qa_sqapt_params(C.Structure):
    _fields_ = [("betas", C.c_void_p), ("gammas", C.c_void_p), ("rungs", C.c_int), ("trotter_slices", C.c_int),
                ("sweeps_per_step", C.c_int), ("worldline_sweeps", C.c_int), ("steps", C.c_int),
                ("swap_interval", C.c_int), ("cluster_sweeps", C.c_int), ("continuous_time_slices", C.c_int),
                ("reads", C.c_int), ("seed", C.c_uint64)]


class qa_sqapt_out(C.Structure):
    _fields_ = [("best_spins", C.c_void_p), ("best_energy", C.c_void_p), ("final_spins", C.c_void_p),
                ("final_energies", C.c_void_p), ("average_energy_trace", C.c_void_p),
                ("swap_acceptance_trace", C.c_void_p)]


class qa_sqaptopt_params(C.Structure):
    _fields_ = [("betas", C.c_void_p), ("gammas", C.c_void_p), ("rungs", C.c_int), ("trotter_slices", C.c_int),
                ("continuous_time_slices", C.c_int), ("sweeps_per_step", C.c_int), ("worldline_sweeps", C.c_int),
                ("cluster_sweeps", C.c_int), ("num_steps", C.c_int), ("swap_interval", C.c_int),
                ("eps_tilde", C.c_double), ("alpha", C.c_double), ("j_perp_end", C.c_double),
                ("calib_probes", C.c_int), ("calib_sweeps", C.c_int), ("reads", C.c_int), ("seed", C.c_uint64)]


class qa_sqaptopt_out(C.Structure):
    _fields_ = [("pt", qa_sqapt_out), ("j_perp_trace", C.c_void_p), ("chi_B_trace", C.c_void_p),
                ("scalars", C.c_void_p)]


class qa_chi_params(C.Structure):
    _fields_ = [("trotter_slices", C.c_int), ("replicas", C.c_int), ("beta", C.c_double),
                ("gamma_start", C.c_double), ("gamma_end", C.c_double), ("num_steps", C.c_int),
                ("sweeps_per_step", C.c_int), ("scan_points", C.c_int), ("scan_sweeps", C.c_int),
                ("scan_burn", C.c_int), ("chi_floor_fraction", C.c_double), ("driver_A0", C.c_double),
                ("beta_ramp_fraction", C.c_double), ("beta_ramp_start", C.c_double), ("reads", C.c_int),
                ("seed", C.c_uint64), ("scan_chi_in", C.c_void_p)]


class qa_chi_out(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in ("best_spins", "best_energy", "energy_trace", "beta_schedule",
                                         "gamma_schedule", "s_schedule", "scan_s", "scan_gamma", "scan_chi_B",
                                         "scalars")]


_lib = None
_lock = threading.Lock()


def load():
    """Load libqa_gpu.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -f qlatanneal_b200/csrc/Makefile` "
                              "(or __graft_entry__.build()).")
        L = C.CDLL(LIB_PATH)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        L.qa_version.restype = C.c_char_p
        L.qa_last_error.argtypes = [C.c_char_p, C.c_size_t]
        L.qa_device_count.argtypes = [C.POINTER(C.c_int)]
        L.qa_create.argtypes = [C.POINTER(vp), i]
        L.qa_destroy.argtypes = [vp]
        L.qa_set_drift_check.argtypes = [vp, d]
        L.qa_set_update_order.argtypes = [vp, i]
        L.qa_get_update_order.argtypes = [vp, C.POINTER(i)]
        L.qa_probe_l2_read.argtypes = [i, C.c_size_t, i, C.POINTER(d)]
        L.qa_set_tuning.argtypes = [vp, C.POINTER(qa_tuning)]
        L.qa_get_tuning.argtypes = [vp, C.POINTER(qa_tuning)]
        L.qa_problem_dense.argtypes = [vp, i, vp, vp, d, C.POINTER(vp)]
        L.qa_problem_qubo.argtypes = [vp, i, vp, vp, vp, C.POINTER(vp)]
        L.qa_problem_sparse.argtypes = [vp, i, vp, i, vp, vp, vp, d, C.POINTER(vp)]
        L.qa_problem_hubo.argtypes = [vp, i, vp, i, vp, vp, vp, d, C.POINTER(vp)]
        L.qa_problem_free.argtypes = [vp]
        L.qa_problem_size.argtypes = [vp, C.POINTER(i)]
        L.qa_sa_run.argtypes = [vp, C.POINTER(vp), i, C.POINTER(qa_sa_params), C.POINTER(qa_run_out),
                                C.POINTER(qa_stats)]
        L.qa_sa_trace_run.argtypes = [vp, C.POINTER(vp), i, C.POINTER(qa_sa_params), C.POINTER(qa_sa_trace),
                                      C.POINTER(qa_run_out), C.POINTER(qa_stats)]
        L.qa_sqa_trace_run.argtypes = [vp, C.POINTER(vp), i, C.POINTER(qa_sqa_params), C.POINTER(qa_sqa_trace),
                                       C.POINTER(qa_run_out), C.POINTER(qa_stats)]
        L.qa_replica_run.argtypes = [vp, C.POINTER(vp), i, C.POINTER(qa_sa_params), C.POINTER(qa_replica_out),
                                     C.POINTER(qa_stats)]
        L.qa_pt_run.argtypes = [vp, C.POINTER(vp), i, C.POINTER(qa_pt_params), C.POINTER(qa_sqapt_out),
                                C.POINTER(qa_stats)]
        L.qa_sqa_run.argtypes = [vp, C.POINTER(vp), i, C.POINTER(qa_sqa_params), C.POINTER(qa_run_out),
                                 C.POINTER(qa_stats)]
        L.qa_sqa_opt_run.argtypes = [vp, C.POINTER(vp), i, C.POINTER(qa_sqaopt_params), C.POINTER(qa_sqaopt_out),
                                     C.POINTER(qa_stats)]
        L.qa_sqapt_run.argtypes = [vp, C.POINTER(vp), i, C.POINTER(qa_sqapt_params), C.POINTER(qa_sqapt_out),
                                   C.POINTER(qa_stats)]
        L.qa_sqapt_opt_run.argtypes = [vp, C.POINTER(vp), i, C.POINTER(qa_sqaptopt_params),
                                       C.POINTER(qa_sqaptopt_out), C.POINTER(qa_stats)]
        L.qa_chi_run.argtypes = [vp, C.POINTER(vp), i, C.POINTER(qa_chi_params), C.POINTER(qa_chi_out),
                                 C.POINTER(qa_stats)]
        L.qa_chi_pilot.argtypes = [vp, C.POINTER(vp), i, C.POINTER(qa_chi_params), vp, C.POINTER(qa_stats)]
        L.qa_mlp_create.argtypes = [vp, C.POINTER(i), i, C.c_uint64, C.POINTER(vp)]
        L.qa_mlp_free.argtypes = [vp]
        L.qa_mlp_num_params.argtypes = [vp, C.POINTER(C.c_int64)]
        L.qa_mlp_get_params.argtypes = [vp, vp, C.c_int64]
        L.qa_mlp_set_params.argtypes = [vp, vp, C.c_int64]
        L.qa_mlp_forward.argtypes = [vp, vp, i, vp]
        L.qa_mlp_loss_grad.argtypes = [vp, vp, vp, i, C.POINTER(C.c_float), vp]
        L.qa_mlp_train_step.argtypes = [vp, vp, vp, i, C.c_float, C.POINTER(C.c_float)]
        for name in list(EXPORTED):
            getattr(L, name)
        _lib = L
        return L


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().qa_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


class FieldDriftError(RuntimeError):
    """The drift check found the incremental float32 local fields farther
    from a float64 recompute than the tolerance (QA_ERR_DRIFT)."""


def check(rc: int) -> None:
    """Map a status code onto the exception qanneal raises for the same failure."""
    if rc == QA_OK:
        return
    msg = last_error()
    if rc == QA_ERR_DRIFT:
        raise FieldDriftError(msg)
    if rc == QA_ERR_ARG:
        raise ValueError(msg)
    if rc == QA_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if rc == QA_ERR_OOM:
        raise MemoryError(msg)
    raise RuntimeError(f"qa_gpu error {rc}: {msg}")


def ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a is not None else None


class Engine:
    """One device context (qa_ctx) per (process, device)."""

    _engines: dict = {}

    def __init__(self, device: int):
        L = load()
        n = C.c_int(0)
        check(L.qa_device_count(C.byref(n)))
        if n.value <= 0:
            raise RuntimeError("no CUDA device is visible: the qlatanneal_b200 engine runs only on a GPU.")
        h = C.c_void_p()
        check(L.qa_create(C.byref(h), int(device)))
        self.L, self.h, self.device = L, h, int(device)

    @classmethod
    def get(cls, device=None) -> "Engine":
        if device is None:
            device = int(os.environ.get("LOCAL_RANK", "0"))
        with _lock:
            e = cls._engines.get(device)
        if e is None:
            e = Engine(device)
            with _lock:
                cls._engines[device] = e
        return e

    def close(self):
        if self.h:
            self.L.qa_destroy(self.h)
            self.h = None
