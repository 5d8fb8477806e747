"""The shuffled spin order of qanneal's SQA sweeps, as the CPU restatement
defines it (test infrastructure; the CUDA engine is checked against it bit for
bit in test_gpu_update_order.py).

qanneal calls std::shuffle on a replica's spin order before every slice,
cluster and worldline sweep (sqa_annealer.cpp:181,216,295;
sqa_parallel_tempering.cpp:209,224,281): a uniformly random permutation.  The
replay model's permutation sorts the spins by Philox keys; these tests pin its
definition and its uniformity.
"""
import math

import numpy as np
from scipy.stats import chi2

DOM_PERM, DOM_SLICE = 13, 3


def _reference_definition(oracle, key, ring, sigma, tag, n):
    keys = []
    for i in range(n):
        if i % 2 == 0:
            ctr = np.array([i >> 1, ring, sigma, ((tag << 8) | DOM_PERM) & 0xFFFFFFFF], np.uint32)
            kk = np.array([key & 0xFFFFFFFF, key >> 32], np.uint32)
            w = [int(x) for x in oracle.philox(ctr, kk)]
        a, b = (w[0], w[1]) if i % 2 == 0 else (w[2], w[3])
        r = (a << 32) | b
        keys.append((r & ~0xFFFFF) | i)
    return [k & 0xFFFFF for k in sorted(keys)]


def test_order_is_the_keyed_sort(oracle):
    for n, key, ring, sigma in [(1, 5, 0, 0), (7, 99, 3, 11), (64, 2 ** 40 + 7, 17, 5), (333, 12345, 2, 1000)]:
        got = oracle.sweep_order(key, ring, sigma, DOM_SLICE, n).tolist()
        assert sorted(got) == list(range(n))
        assert got == _reference_definition(oracle, key, ring, sigma, DOM_SLICE, n)


def test_order_is_uniform_over_permutations(oracle):
    """n = 4: all 24 orders equally likely (chi-square over 24 000 sweeps)."""
    n, draws = 4, 24000
    counts = {}
    for s in range(draws):
        o = tuple(oracle.sweep_order(777, 3, s, DOM_SLICE, n).tolist())
        counts[o] = counts.get(o, 0) + 1
    assert len(counts) == math.factorial(n)
    exp_c = draws / math.factorial(n)
    stat = sum((c - exp_c) ** 2 / exp_c for c in counts.values())
    assert chi2.sf(stat, math.factorial(n) - 1) > 1e-4


def test_order_positions_are_uniform(oracle):
    """n = 40: every spin lands in each quarter of the order equally often
    (chi-square over 4000 sweeps), and orders of different rings and sweeps
    differ."""
    n, draws = 40, 4000
    hist = np.zeros((n, 4))
    seen = set()
    for s in range(draws):
        o = oracle.sweep_order(2024, s % 7, s, DOM_SLICE, n)
        seen.add(tuple(o.tolist()))
        pos = np.empty(n, int)
        pos[o] = np.arange(n)
        hist[np.arange(n), pos * 4 // n] += 1
    assert len(seen) == draws
    stat = float(((hist - draws / 4) ** 2 / (draws / 4)).sum())
    assert chi2.sf(stat, n * 3) > 1e-4


def test_order_switch(oracle):
    assert oracle.update_order() == "reference"
    oracle.set_update_order("checkerboard")
    try:
        assert oracle.update_order() == "checkerboard"
    finally:
        oracle.set_update_order("reference")
