"""SQA-Chi restatement pins (CPU).

* Stage 2 (schedule from a chi_B scan) equals qanneal's bit for bit: the
  reference's own run_chi output curve is fed to the restatement.
* tests/test_sqa_chi_annealer.cpp's checks hold for the restated run_chi:
  schedule structure on the xorshift SK instance, exact ground states of a
  dense ferromagnetic chain (-11) and a sparse ring (-12), degenerate range.
"""
import numpy as np
import pytest

M64 = (1 << 64) - 1


def xorshift_sk(n):
    """make_sk_problem (tests/test_sqa_chi_annealer.cpp:36-52)."""
    s = 0x9E3779B97F4A7C15
    J = np.zeros((n, n))
    for i in range(n):
        for j in range(i + 1, n):
            s ^= (s << 13) & M64
            s ^= s >> 7
            s ^= (s << 17) & M64
            w = ((s % 100000) / 100000.0 - 0.5) * 2.0
            J[i, j] = J[j, i] = w
    return np.zeros(n), J


def ferro_chain(n):
    J = np.zeros((n, n))
    for i in range(n - 1):
        J[i, i + 1] = J[i + 1, i] = -1.0
    return np.zeros(n), J


def test_stage2_bitwise_against_reference(oracle, ref):
    h, J = xorshift_sk(10)
    r = ref.dense(h, J).chi_run(8, 4, 4.0, 4.0, 0.05, 120, 8, 12, 24, 8, 2026)
    b, g, s, sc = oracle.chi_schedule(r["scan_s"], r["scan_gamma"], r["scan_chi"], 4.0, 4.0, 0.05, 4.0, 8, 120)
    np.testing.assert_array_equal(b, r["beta"])
    np.testing.assert_array_equal(g, r["gamma"])
    np.testing.assert_array_equal(s, r["s"])
    np.testing.assert_array_equal(sc[:4], r["scalars"][:4])
    o = oracle.chi_run(oracle.dense(h, J), 8, 4, 4.0, 4.0, 0.05, 120, 8, 12, 24, 8, 5)
    np.testing.assert_array_equal(o["scan_s"], r["scan_s"])
    np.testing.assert_array_equal(o["scan_gamma"], r["scan_gamma"])
    # a flat (degenerate) curve falls back to a linear-in-s schedule in both
    flat = np.zeros(12)
    b2, g2, s2, sc2 = oracle.chi_schedule(r["scan_s"], r["scan_gamma"], flat, 4.0, 4.0, 0.05, 4.0, 8, 50)
    assert sc2[3] == 1.0 and np.all(np.diff(s2[15:]) > 0)


def test_reference_chi_checks_on_restatement(oracle):
    # (A) diagnostics and schedule structure (test_sqa_chi_annealer.cpp:71-143)
    h, J = xorshift_sk(10)
    res = oracle.chi_run(oracle.dense(h, J), 8, 4, 4.0, 4.0, 0.05, 120, 8, 12, 24, 8, 2026)
    chi = res["scan_chi"]
    assert np.all(chi >= 0.0) and chi.max() > chi.min()
    s_star, g_star, jp_star, floor_, A0 = res["scalars"]
    assert res["scan_s"][0] <= s_star <= res["scan_s"][-1]
    assert 0.05 - 1e-9 <= g_star <= 4.0 + 1e-9 and jp_star > 0.0 and floor_ > 0.0 and A0 == 4.0
    g = res["gamma"]
    assert np.all(np.diff(g) <= 1e-12) and abs(g[0] - 4.0) < 1e-9 and abs(g[-1] - 0.05) < 1e-6
    s = res["s"]
    assert np.all(np.diff(s) >= -1e-12)
    ds = np.diff(s)
    mid = 0.5 * (s[1:] + s[:-1])
    win = 0.15 * (res["scan_s"][-1] - res["scan_s"][0])
    keep = ds > 0
    near = keep & (np.abs(mid - s_star) < win)
    assert near.sum() > 0 and ds[near].mean() <= ds[keep].mean() * 1.05
    # (B) dense ferromagnetic chain, exact ground state -11 (:145-159)
    h, J = ferro_chain(12)
    assert oracle.chi_run(oracle.dense(h, J), 8, 4, 4.0, 3.0, 0.05, 100, 10, 10, 20, 6, 7)["best_energy"] == -11.0
    # (C) sparse ferromagnetic ring, -12 (:161-175)
    ring = [(i, (i + 1) % 12, -1.0) for i in range(12)]
    assert oracle.chi_run(oracle.sparse(12, np.zeros(12), ring), 8, 4, 4.0, 3.0, 0.05, 100, 10, 10, 20, 6,
                          11)["best_energy"] == -12.0
    # (D) degenerate tiny range (:177-192)
    h, J = ferro_chain(6)
    res = oracle.chi_run(oracle.dense(h, J), 4, 2, 0.5, 0.2, 0.15, 20, 4, 4, 4, 2, 3)
    assert len(res["gamma"]) == 20 and np.all(np.isfinite(res["gamma"])) and np.all(res["gamma"] > 0)


def _ci95(x):
    x = np.asarray(x, float)
    return x.mean(), 1.96 * x.std(ddof=1) / np.sqrt(len(x))


def test_chi_restatement_matches_reference_statistics(oracle, ref):
    """Mean chi_B curve and final production energy inside 95% CIs."""
    h, J = xorshift_sk(12)
    m, rm = oracle.dense(h, J), ref.dense(h, J)
    args = (6, 2, 3.0, 3.0, 0.1, 20, 3, 6, 12, 4)
    co, cr, eo, er = [], [], [], []
    for k in range(150):
        o = oracle.chi_run(m, *args, 500 + k)
        r = rm.chi_run(*args, 9000 + k)
        co.append(o["scan_chi"].sum()); cr.append(r["scan_chi"].sum())
        eo.append(o["trace"][-1]); er.append(r["trace"][-1])
    for a, b in ((co, cr), (eo, er)):
        (ma, ca), (mb, cb) = _ci95(a), _ci95(b)
        assert abs(ma - mb) <= 1.5 * (ca + cb), (ma, ca, mb, cb)
