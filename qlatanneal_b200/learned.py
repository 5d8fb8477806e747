"""Learned chi_B(Gamma) curves for SQA-Chi: instance features -> predicted curve.

run_chi spends its pilot stage (sqa_chi_annealer.cpp:217-281) measuring the
susceptibility chi_B at scan_points values of s = A0/(A0+Gamma) before it can
build the schedule.  ChiCurveModel predicts that curve from 16 features of the
instance and the run parameters, so the production anneal can start at once;
when the network's own predicted uncertainty is high it returns None and the
pilot runs as before.

Training data come from the plain pilot (``pilot_curves``), training and
inference run on the GPU through the MLP kernels of libqa_gpu.so
(qa_mlp_*: bfloat16 weights, float32 accumulation, Adam).  Targets are curve
shapes y = ln(chi / max chi + 0.01): the schedule construction only depends on
the shape (its floor is relative and its CDF is normalised).
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from .annealers import _random_seed
from .models import DenseIsing, HigherOrderIsing, SparseIsing

N_FEATURES = 16
TARGET_EPS = 0.01
FEATURE_NAMES = [
    "log_n", "density", "degree_cv", "mean_abs_J", "rms_J", "max_abs_J", "mean_J", "log_degree",
    "mean_abs_h", "rms_h", "lambda_over_rms_sqrt_deg", "lambda_over_n", "beta", "log_gamma_start",
    "log_gamma_end", "slices",
]


def _two_body(ising):
    """(n, upper-triangle coupling values, degrees, h, matvec) of the two-body
    part; matvec(x) = J x with the full symmetric J."""
    n = ising.size()
    if isinstance(ising, DenseIsing):
        J = np.array(ising.couplings(), dtype=np.float64)
        np.fill_diagonal(J, 0.0)
        nz = J != 0.0
        deg = nz.sum(axis=1).astype(float)
        v = J[np.triu(nz, 1)]
        return n, v, deg, np.asarray(ising.fields(), float), (lambda x: J @ x)
    if isinstance(ising, SparseIsing):
        r, c, v = ising._ei, ising._ej, ising._w
        h = np.asarray(ising._h, float)
    elif isinstance(ising, HigherOrderIsing):
        rs, cs, vs = [], [], []
        for k, w in ising.terms():
            for a in range(len(k)):
                for b in range(a + 1, len(k)):
                    rs.append(k[a]); cs.append(k[b]); vs.append(w)
        r, c, v = np.asarray(rs, int), np.asarray(cs, int), np.asarray(vs, float)
        h = np.asarray(ising.h(), float)
    else:
        raise TypeError("unsupported model")
    rows, cols, vals = np.concatenate([r, c]), np.concatenate([c, r]), np.concatenate([v, v])
    deg = np.bincount(rows, minlength=n).astype(float)
    return n, np.asarray(v, float), deg, h, (lambda x: np.bincount(rows, weights=vals * x[cols], minlength=n))


def _top_eigenvalue(n: int, matvec, iters: int = 100) -> float:
    """Largest |eigenvalue| of the symmetric coupling matrix by power
    iteration; the estimate is |J x| for the unit iterate x, which tends to
    |lambda_max| even when -lambda_max is (almost) as large, as in the
    symmetric spectra of random +-1 couplings."""
    x = np.cos(np.arange(n) * 0.7 + 0.3)
    x /= np.linalg.norm(x)
    nrm = 0.0
    for _ in range(iters):
        y = matvec(x)
        nrm = float(np.linalg.norm(y))
        if nrm == 0.0:
            return 0.0
        x = y / nrm
    return nrm


def instance_features(ising, beta: float, gamma_start: float, gamma_end: float, slices: int) -> np.ndarray:
    """The 16 inputs of the network: size, degree mean and spread, coupling
    moments, field moments, the top eigenvalue of J (power iteration), and
    the run parameters (beta, Gamma range, Trotter slices)."""
    n, v, deg, h, matvec = _two_body(ising)
    mdeg = max(float(deg.mean()), 1e-9)
    av = np.abs(v)
    rms = float(np.sqrt(np.mean(v * v))) if v.size else 0.0
    lam = _top_eigenvalue(n, matvec) if v.size else 0.0
    return np.array([
        math.log(n) / 8.0,
        mdeg / n,
        float(deg.std()) / mdeg,
        float(av.mean()) if v.size else 0.0,
        rms,
        float(av.max()) if v.size else 0.0,
        float(v.mean()) if v.size else 0.0,
        math.log(mdeg + 1.0) / 8.0,
        float(np.abs(h).mean()),
        float(np.sqrt(np.mean(h * h))),
        lam / max(rms * math.sqrt(mdeg), 1e-9),
        lam / n,
        beta / 10.0,
        math.log(gamma_start),
        math.log(gamma_end),
        slices / 64.0,
    ])


def curve_target(chi: np.ndarray) -> np.ndarray:
    chi = np.maximum(np.asarray(chi, float), 0.0)
    m = chi.max(axis=-1, keepdims=True)
    return np.log(np.where(m > 0, chi / np.where(m > 0, m, 1.0), 0.0) + TARGET_EPS)


def target_curve(y: np.ndarray) -> np.ndarray:
    return np.maximum(np.exp(np.asarray(y, float)) - TARGET_EPS, 0.0)


def pilot_curves(isings: Sequence, beta: float, gamma_start: float, gamma_end: float, slices: int, points: int = 64,
                 sweeps: int = 200, burn: int = 50, replicas: int = 1, reads: int = 1, seed: int = 0,
                 average: bool = True, device: Optional[int] = None) -> np.ndarray:
    """chi_B curves of the plain pilot (run_chi Stage 1) of every instance, all
    instances of one model kind in one GPU call; read r uses the key seed + r.
    Returns [instances][points], the mean over the reads, or with
    ``average=False`` every read's curve, [instances][reads][points]."""
    eng = _lib.Engine.get(device)
    out = np.zeros((len(isings), int(reads), int(points)))
    groups: Dict[str, List[int]] = {}
    for i, m in enumerate(isings):
        groups.setdefault(m.kind, []).append(i)
    prm = _lib.qa_chi_params(int(slices), int(replicas), float(beta), float(gamma_start), float(gamma_end), 2, 1,
                             int(points), int(sweeps), int(burn), 1e-6, 0.0, 0.3, 0.1, int(reads), int(seed), None)
    for idx in groups.values():
        probs = (C.c_void_p * len(idx))(*[isings[i]._device_problem(eng) for i in idx])
        chi = np.zeros(len(idx) * int(reads) * int(points))
        _lib.check(eng.L.qa_chi_pilot(eng.h, probs, len(idx), C.byref(prm), chi.ctypes.data, None))
        out[idx] = chi.reshape(len(idx), int(reads), int(points))
    return out.mean(axis=1) if average else out


def schedule_distance(chi_a: np.ndarray, chi_b: np.ndarray, floor_fraction: float = 1e-6) -> np.ndarray:
    """Kolmogorov distance between the schedules two chi_B curves give: the
    largest gap between the normalised cumulative weights max(chi, floor) over
    the s grid (run_chi places its steps at the quantiles of that CDF)."""
    def cdf(c):
        c = np.maximum(np.asarray(c, float), 0.0)
        w = np.maximum(c, np.maximum(floor_fraction * c.max(axis=-1, keepdims=True), 1e-12))
        q = np.cumsum(w, axis=-1)
        return q / q[..., -1:]
    return np.abs(cdf(chi_a) - cdf(chi_b)).max(axis=-1)


class ChiCurveModel:
    """MLP features(16) -> [mean | log-variance] of the 64-point curve shape.

    ``run_params`` = dict(beta, gamma_start, gamma_end, slices, points) of the
    pilot scans it was trained on; calling the model on an instance returns the
    predicted chi_B curve for those run parameters (the ``chi_curve`` argument of
    solve()), or None -- run the pilot -- when the prediction is not to be
    trusted: the mean predicted standard deviation exceeds ``max_std`` (by
    default calibrated by ``fit`` to twice the 95th percentile over the
    training set), or a feature lies more than ``max_z`` training standard
    deviations from the training mean (an instance unlike any it was trained on).
    """

    def __init__(self, points: int = 64, hidden: Sequence[int] = (128, 128, 128), seed: Optional[int] = None,
                 device: Optional[int] = None, max_std: Optional[float] = None, max_z: float = 4.0):
        self.points = int(points)
        self.dims = [N_FEATURES] + [int(h) for h in hidden] + [2 * self.points]
        self.device = device
        self.max_std = None if max_std is None else float(max_std)
        self._calibrate_std = max_std is None
        self.max_z = float(max_z)
        self.last_std = self.last_z = float("nan")
        self.mu = np.zeros(N_FEATURES)
        self.sd = np.ones(N_FEATURES)
        self.run_params: Dict[str, float] = {}
        eng = _lib.Engine.get(device)
        self._eng = eng
        h = C.c_void_p()
        d = (C.c_int * len(self.dims))(*self.dims)
        _lib.check(eng.L.qa_mlp_create(eng.h, d, len(self.dims), int(_random_seed() if seed is None else seed),
                                       C.byref(h)))
        self._h = h
        cnt = C.c_int64()
        _lib.check(eng.L.qa_mlp_num_params(h, C.byref(cnt)))
        self.n_params = int(cnt.value)

    def __del__(self):
        try:
            if self._h:
                self._eng.L.qa_mlp_free(self._h)
                self._h = None
        except Exception:
            pass

    # ---- parameters
    def get_params(self) -> np.ndarray:
        p = np.zeros(self.n_params, np.float32)
        _lib.check(self._eng.L.qa_mlp_get_params(self._h, p.ctypes.data, self.n_params))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        _lib.check(self._eng.L.qa_mlp_set_params(self._h, p.ctypes.data, self.n_params))

    def save(self, path: str) -> None:
        np.savez(path, params=self.get_params(), mu=self.mu, sd=self.sd, dims=np.asarray(self.dims),
                 max_std=np.nan if self.max_std is None else self.max_std, max_z=self.max_z,
                 **{"rp_" + k: v for k, v in self.run_params.items()})

    @classmethod
    def load(cls, path: str, device: Optional[int] = None) -> "ChiCurveModel":
        z = np.load(path)
        dims = [int(x) for x in z["dims"]]
        ms = float(z["max_std"])
        m = cls(points=dims[-1] // 2, hidden=dims[1:-1], seed=0, device=device,
                max_std=None if math.isnan(ms) else ms, max_z=float(z["max_z"]))
        m.set_params(z["params"])
        m.mu, m.sd = z["mu"], z["sd"]
        m.run_params = {k[3:]: float(z[k]) for k in z.files if k.startswith("rp_")}
        return m

    # ---- training / inference (GPU kernels)
    def _norm(self, X: np.ndarray) -> np.ndarray:
        return np.ascontiguousarray((np.asarray(X, float) - self.mu) / self.sd, np.float32)

    def loss_grad(self, X: np.ndarray, Y: np.ndarray) -> Tuple[float, np.ndarray]:
        Xn = self._norm(X)
        T = np.ascontiguousarray(Y, np.float32)
        loss = C.c_float()
        g = np.zeros(self.n_params, np.float32)
        _lib.check(self._eng.L.qa_mlp_loss_grad(self._h, Xn.ctypes.data, T.ctypes.data, len(Xn), C.byref(loss),
                                                g.ctypes.data))
        return float(loss.value), g

    def loss(self, X: np.ndarray, Y: np.ndarray) -> float:
        Xn = self._norm(X)
        T = np.ascontiguousarray(Y, np.float32)
        loss = C.c_float()
        _lib.check(self._eng.L.qa_mlp_loss_grad(self._h, Xn.ctypes.data, T.ctypes.data, len(Xn), C.byref(loss),
                                                None))
        return float(loss.value)

    def fit(self, X: np.ndarray, Y: np.ndarray, epochs: int = 300, batch: int = 64, lr: float = 2e-3,
            seed: int = 0, run_params: Optional[Dict[str, float]] = None, val_fraction: float = 0.15,
            patience: int = 30) -> List[float]:
        """Adam on the GPU with a cosine learning rate; keeps the parameters of
        the epoch with the lowest loss on a held-out ``val_fraction`` of the
        samples (pilot curves are noisy targets: training past that point fits
        their noise) and stops after ``patience`` epochs without improvement.
        Returns the training loss per epoch."""
        X = np.asarray(X, float)
        Y = np.asarray(Y, np.float32)
        self.mu = X.mean(0)
        self.sd = np.maximum(X.std(0), 1e-6)
        if run_params:
            self.run_params = dict(run_params)
        rng = np.random.default_rng(seed)
        perm = rng.permutation(len(X))
        n_val = int(round(val_fraction * len(X))) if len(X) >= 10 else 0
        val, tr = perm[:n_val], perm[n_val:]
        Xn = self._norm(X[tr])
        Yt = Y[tr]
        hist: List[float] = []
        best_val, best_p, since = float("inf"), None, 0
        loss = C.c_float()
        for ep in range(epochs):
            order = rng.permutation(len(Xn))
            tot = 0.0
            cur_lr = max(lr * 0.5 * (1 + math.cos(math.pi * ep / max(epochs, 1))), 1e-5)
            for b0 in range(0, len(Xn), batch):
                sel = order[b0:b0 + batch]
                xb = np.ascontiguousarray(Xn[sel])
                yb = np.ascontiguousarray(Yt[sel])
                _lib.check(self._eng.L.qa_mlp_train_step(self._h, xb.ctypes.data, yb.ctypes.data, len(sel),
                                                         C.c_float(cur_lr), C.byref(loss)))
                tot += loss.value * len(sel)
            hist.append(tot / len(Xn))
            if n_val:
                v = self.loss(X[val], Y[val])
                if v < best_val:
                    best_val, best_p, since = v, self.get_params(), 0
                else:
                    since += 1
                    if since >= patience:
                        break
        if best_p is not None:
            self.set_params(best_p)
        self.val_loss = best_val
        if self._calibrate_std:
            _, std = self.predict(X)
            self.max_std = 2.0 * float(np.quantile(std.mean(axis=1), 0.95))
        return hist

    def predict(self, X: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
        Xn = self._norm(np.atleast_2d(X))
        Yo = np.zeros((len(Xn), 2 * self.points), np.float32)
        _lib.check(self._eng.L.qa_mlp_forward(self._h, Xn.ctypes.data, len(Xn), Yo.ctypes.data))
        mean = Yo[:, :self.points].astype(float)
        std = np.exp(0.5 * np.clip(Yo[:, self.points:], -12, 12)).astype(float)
        return mean, std

    def curve(self, ising, beta=None, gamma_start=None, gamma_end=None, slices=None,
              points: Optional[int] = None) -> Optional[np.ndarray]:
        """Predicted chi_B curve on the pilot's s grid (linear in s from
        s(gamma_start) to s(gamma_end)), resampled to ``points`` values; None
        when the prediction is not trusted (see the class docstring)."""
        rp = self.run_params
        f = instance_features(ising, beta if beta is not None else rp["beta"],
                              gamma_start if gamma_start is not None else rp["gamma_start"],
                              gamma_end if gamma_end is not None else rp["gamma_end"],
                              slices if slices is not None else rp["slices"])
        mean, std = self.predict(f)
        self.last_std = float(std.mean())
        self.last_z = float(np.max(np.abs(f - self.mu) / self.sd))
        if self.last_z > self.max_z:
            return None
        if self.max_std is not None and self.last_std > self.max_std:
            return None
        c = target_curve(mean[0])
        c = c / c.max() if c.max() > 0 else np.ones_like(c)
        if points is not None and int(points) != self.points:
            c = np.interp(np.linspace(0.0, 1.0, int(points)), np.linspace(0.0, 1.0, self.points), c)
        return c

    __call__ = curve


def synthetic_instances(count: int, n_min: int, n_max: int, seed: int, kinds=("sk", "regular3")):
    """Seeded training instances: alternately dense Sherrington-Kirkpatrick
    (J in {-1,+1}) and random 3-regular (J in {-1,+1}), h = 0, n uniform in
    [n_min, n_max] (even)."""
    from .instances import regular3, sk_dense
    rng = np.random.default_rng(seed)
    for i in range(count):
        n = int(rng.integers(n_min // 2, n_max // 2 + 1)) * 2
        s = int(rng.integers(1 << 31))
        kind = kinds[i % len(kinds)]
        if kind == "sk":
            h, J = sk_dense(n, s)
            yield DenseIsing(h, J)
        else:
            h, e = regular3(n, s, h_choices=(0.0,))
            yield SparseIsing(h, e, n)


def training_set(models, beta: float, gamma_start: float, gamma_end: float, slices: int, points: int = 64,
                 sweeps: int = 200, burn: int = 50, reads: int = 1, seed: int = 0, chunk: int = 64,
                 device: Optional[int] = None) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """(features [N][16], targets [N][points], pilot curves [N][points]) for a
    stream of models, piloted ``chunk`` at a time (their device copies are
    freed after each chunk)."""
    X, chi = [], []
    batch = []

    def flush():
        if not batch:
            return
        chi.append(pilot_curves(batch, beta, gamma_start, gamma_end, slices, points, sweeps, burn,
                                reads=reads, seed=seed, device=device))
        for m in batch:
            X.append(instance_features(m, beta, gamma_start, gamma_end, slices))
            m.release()
        batch.clear()

    for m in models:
        batch.append(m)
        if len(batch) >= chunk:
            flush()
    flush()
    C_ = np.concatenate(chi) if chi else np.zeros((0, points))
    return np.asarray(X), curve_target(C_), C_
