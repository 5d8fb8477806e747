"""The sweep kernels' pre-test of a Metropolis proposal (metropolis_maybe24 in
qa_device.cuh) never rejects a move that the exact test accepts.

The exact test accepts iff u24 < det_expf(y) * 2^24 (qanneal's
u < exp(-dE), annealer.cpp:55, sqa_annealer.cpp:198, with the deterministic
float32 exponential).  The pre-test answers "maybe" iff
bits(u24) < ceil(fma(y, log2(e) 2^23, 151.001 * 2^23)).  Both are monotone in
u24, so it suffices that the largest accepted u24 of each y passes the
pre-test; this checks that with the oracle's det_expf, and that the slack stays
far above the pre-test's own rounding (the fused multiply-add is restated in
float64, within one float32 ulp of the device's)."""
import math

import numpy as np
import pytest

C = float(np.float32(1.44269504) * np.float32(8388608.0))
D = float(np.float32(151.001) * np.float32(8388608.0))


def pretest_K(y: float) -> int:
    return math.ceil(float(np.float32(float(np.float32(y)) * C + D)))


def bits(u: float) -> int:
    return int(np.array(u, np.float32).view(np.int32))


def largest_accepted_u24(oracle, y: float):
    e = oracle.expf(float(np.float32(y))) * 16777216.0  # exact scaling of a float32
    if y >= 0.0:
        return 16777215.0
    if y <= -17.0 or e <= 0.0:
        return None
    u = math.ceil(e) - 1.0  # u24 values are integers 0 .. 2^24 - 1
    return min(u, 16777215.0) if u >= 0.0 else None


def _ys():
    rng = np.random.default_rng(5)
    ys = [rng.uniform(-17.0, 0.0, 40000), rng.uniform(-1e-3, 0.0, 2000), rng.uniform(-17.0, -16.9, 2000)]
    # around the points where k = rint(y log2 e) changes
    half = (np.arange(-25, 1) + 0.5) / 1.4426950408889634
    ys.append((half[:, None] + rng.uniform(-1e-5, 1e-5, (len(half), 40))).ravel())
    ys.append(np.array([0.0, -0.0, -1e-30, -16.999998, -17.0, 1.0, 30.0]))
    y = np.concatenate(ys).astype(np.float32)
    return y[(y > -17.0)]


def test_pretest_never_rejects_an_accepted_move(oracle):
    worst = math.inf
    for y in _ys():
        u = largest_accepted_u24(oracle, float(y))
        if u is None:
            continue
        K = pretest_K(float(y))
        assert bits(u) < K, (float(y), u, K)
        worst = min(worst, (K - bits(u)) / 8388608.0)
    # slack in log2 units: the 0.001 margin less the bound's own looseness
    assert worst > 5e-4


@pytest.mark.parametrize("y", [-0.5, -3.0, -9.25, -16.0])
def test_pretest_rejects_most_rejections(oracle, y):
    """The pre-test is sharp: it passes at most ~7% more uniforms than the
    exact test accepts (the linear log2 of the float bits is within 0.087)."""
    u_max = largest_accepted_u24(oracle, y)
    K = pretest_K(y)
    passed = sum(1 for u in np.linspace(0, 16777215, 20001) if bits(float(u)) < K)
    accepted = sum(1 for u in np.linspace(0, 16777215, 20001) if u <= u_max)
    assert accepted <= passed <= 1.07 * accepted + 2
