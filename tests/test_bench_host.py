"""Host logic of bench.py (no GPU): the committed DRAM-traffic figure it
reports, the field-cache model of algorithmic bytes, the TTS99 formula and
the reference arm's sample description."""
import math
import os
import sys
from types import SimpleNamespace

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def test_traffic_figure_parses():
    t = bench.load_traffic()
    assert t is not None and t > 0
    # the figure is the per-anneal scale-up of a three-launch capture
    assert t == pytest.approx(569003 * 1280, rel=1e-3)


def test_algorithmic_bytes_model():
    st = SimpleNamespace(slice_attempts=1000, worldline_attempts=10, slice_accepts=7, worldline_accepts=1)
    P, n = 32, 512
    att = 1000 + 10 * P
    acc = 7 + 1 * P
    assert bench.algorithmic_bytes(st, n, P) == acc * n + att * (4.0 + 3.0 / 8.0)
    assert bench.site_attempts(st, P) == att


def test_tts99():
    assert bench.tts99(1.0, 100, 0.0) == float("inf")
    assert bench.tts99(1.0, 100, 0.995) == pytest.approx(0.01)
    p = 0.02
    assert bench.tts99(2.0, 512, p) == pytest.approx(2.0 / 512 * math.log(0.01) / math.log(1.0 - p))


def test_bench_workload_is_the_configured_one():
    assert bench.WL["n"] == 512 and bench.WL["P"] == 32 and bench.WL["reads"] == 256 and bench.WL["steps"] == 1000
    betas, gammas = bench.schedule()
    assert len(betas) == 1000 and betas[0] == 0.5 * 32
    assert gammas[0] == 3.0 and gammas[-1] == pytest.approx(0.01)
