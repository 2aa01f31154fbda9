"""CPU tests of the oracle (oracle/oracle.c): pinned against the reference's
golden vectors (rust/src/peaks.rs:290-371) and known-answer tests
(tests/test_periodfind.py:468-484, 580-595, 656-671, 731-752), plus the
structural properties the reference relies on."""

import json
import os

import numpy as np
import pytest

import lightcurves as lc

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "peaks_golden.json")


def _golden_cases():
    with open(GOLDEN) as fh:
        return json.load(fh)["cases"]


@pytest.mark.parametrize("case", _golden_cases(), ids=lambda c: c["name"])
def test_peaks_golden(oracle, case):
    idx, val = oracle.find_top_peaks(case["data"], case["n_peaks"], case["min_distance"],
                                     case["use_max"])
    if case["expect_idx"] is not None:
        assert idx.tolist() == case["expect_idx"]
        np.testing.assert_array_equal(val, np.array(case["expect_val"], np.float32))
    if case["name"] == "respects_n_peaks_limit":
        assert val[0] > val[1]
    if case["name"] == "chunked_matches_single_pass":
        # peaks.rs:337-355 splits the scan at 50 and expects the same answer
        # as one pass; the oracle's single pass must yield sorted maxima.
        assert len(idx) == 5 and np.all(np.diff(val) <= 0)


def test_peaks_batched_padding(oracle):
    data = np.zeros((2, 7, 1), np.float32)
    data[0, 3, 0] = 1.0
    idx, val = oracle.find_top_peaks_batched(data, 4, 1, True)
    assert idx.tolist() == [[3, -1, -1, -1], [-1, -1, -1, -1]]
    assert val.tolist() == [[1.0, 0.0, 0.0, 0.0], [0.0] * 4]


def test_peaks_ties_prefer_lower_index(oracle):
    data = [0, 2, 0, 2, 0, 2, 0, 1, 0]
    idx, val = oracle.find_top_peaks(data, 2, 1, True)
    assert idx.tolist() == [1, 3]


def test_peaks_min_distance_monotone(oracle):
    t, m = lc.sine_curve(3.0, n=500)
    pg = oracle.aov([t], [m], np.linspace(1, 10, 500, dtype=np.float32),
                    np.zeros(1, np.float32), 10)[0].ravel()
    close, _ = oracle.find_top_peaks(pg, 32, 1, True)
    far, _ = oracle.find_top_peaks(pg, 32, 20, True)
    assert len(far) <= len(close)


@pytest.mark.parametrize("algo", ["ce", "aov", "ls"])
def test_known_period(oracle, algo):
    true_p = 5.0
    t, m = lc.sine_curve(true_p, n=800, noise=0.02, t_span=200.0)
    periods = lc.trial_periods(true_p, n=500)
    pdts = np.zeros(1, np.float32)
    if algo == "ce":
        pg = oracle.ce([t], [lc.normalize(m)], periods, pdts, 15, 10)[0, :, 0]
        best = periods[np.argmin(pg)]
    elif algo == "aov":
        pg = oracle.aov([t], [m], periods, pdts, 15)[0, :, 0]
        best = periods[np.argmax(pg)]
    else:
        pg = oracle.ls([t], [lc.center(m)], periods, pdts)[0, :, 0]
        best = periods[np.argmax(pg)]
    assert abs(best - true_p) / true_p < 0.05


def test_fused_tcorr_matches_at_zero_pdt(oracle):
    t, m = lc.sine_curve(2.0, n=300)
    periods = np.linspace(0.5, 5, 300, dtype=np.float32)
    pdts = np.zeros(1, np.float32)
    a = oracle.ce([t], [lc.normalize(m)], periods, pdts, fused_tcorr=False)
    b = oracle.ce([t], [lc.normalize(m)], periods, pdts, fused_tcorr=True)
    np.testing.assert_array_equal(a, b)


def test_empty_curve_values(oracle):
    """The reference CPU path on an empty curve: CE is NaN (0/0 probabilities),
    AOV and LS return 0 (rust/src/aov.rs:197-198, rust/src/ls.rs:276-277)."""
    e = np.zeros(0, np.float32)
    periods = np.array([1.0, 2.0, 3.0], np.float32)
    pdts = np.zeros(1, np.float32)
    assert np.all(np.isnan(oracle.ce([e], [e], periods, pdts)))
    assert np.all(oracle.aov([e], [e], periods, pdts) == 0)
    assert np.all(oracle.ls([e], [e], periods, pdts) == 0)


def test_counts_sum_and_overlap(oracle):
    t, m = lc.sine_curve(2.0, n=257)
    mn = lc.normalize(m)
    _, c1 = oracle.ce_counts(t, mn, 2.0, 0.0, 10, 10, 1, 1)
    assert c1.sum() == 257
    _, c3 = oracle.ce_counts(t, mn, 2.0, 0.0, 10, 10, 3, 2)
    assert c3.sum() == 257 * 6
    _, a2 = oracle.aov_counts(t, m, 2.0, 0.0, 15, 2)
    assert a2.sum() == 257 * 2


def test_ls_f32_close_to_f64(oracle):
    t, m = lc.sine_curve(3.0, n=400, t_span=100.0)
    periods = np.linspace(1, 10, 200, dtype=np.float32)
    pdts = np.zeros(1, np.float32)
    a = oracle.ls([t], [lc.center(m)], periods, pdts)
    b = oracle.ls_f64([t], [lc.center(m)], periods, pdts)
    np.testing.assert_allclose(a, b, rtol=1e-3, atol=1e-3)


def test_batched_equals_per_curve(oracle):
    curves = [lc.sine_curve(p, n=n, seed=s) for s, (p, n) in enumerate([(2, 10), (3, 33), (4, 1)])]
    ts = [c[0] for c in curves]
    ms = [lc.normalize(c[1]) if len(c[1]) > 1 else c[1] for c in curves]
    periods = np.linspace(1, 5, 40, dtype=np.float32)
    pdts = np.array([0.0, 1e-3], np.float32)
    allb = oracle.ce(ts, ms, periods, pdts)
    for i in range(3):
        one = oracle.ce([ts[i]], [ms[i]], periods, pdts)
        np.testing.assert_array_equal(allb[i], one[0])


def _fpw_numpy(t, m, e, periods, pdts, n_bins):
    """FPW from numpy: the fold and the f32 bin rule of rust/src/fpw.rs:41-44,
    the bin sums and the statistic in float64 (fpw.rs:46-63)."""
    t64 = t.astype(np.float64)
    w = (1.0 / (e.astype(np.float64) ** 2)) if e is not None else np.ones(len(t))
    out = np.zeros((len(periods), len(pdts)))
    for pi, P in enumerate(periods):
        for di, dt in enumerate(pdts):
            corr = np.float32(np.float32(dt) / np.float32(P)) / np.float32(2.0)
            r = (t64 - np.float64(corr) * t64 * t64) / np.float64(P)
            phase = np.abs(r - np.floor(r)).astype(np.float32)
            b = np.minimum((phase * np.float32(n_bins)).astype(np.int64), n_bins - 1)
            V = np.bincount(b, weights=w, minlength=n_bins)
            Y = np.bincount(b, weights=w * m.astype(np.float64), minlength=n_bins)
            ok = V > 0
            out[pi, di] = np.sum(Y[ok] ** 2 / (2 * V[ok]))
    return out


def test_fpw_matches_numpy_restatement(oracle):
    """The oracle's FPW (f32 sums in point order, as rust/src/fpw.rs) is within
    f32 rounding of the same statistic summed in float64."""
    rng = np.random.default_rng(3)
    t = lc.uniform_times(rng, 700, 300.0)
    m = lc.noisy(rng, lc.sinusoid(t, 3.7, amp=0.4, offset=15.0), 0.05)
    e = rng.uniform(0.02, 0.2, 700).astype(np.float32)
    P = lc.trial_periods(3.7, n=60)
    D = np.array([0.0, 1e-4], np.float32)
    for errs, nb in ((None, 10), ([e], 20), ([e], 7)):
        got = oracle.fpw([t], [m], P, D, nb, errs=errs)[0]
        want = _fpw_numpy(t, m, None if errs is None else e, P, D, nb)
        np.testing.assert_allclose(got, want, rtol=2e-5)


def test_fpw_one_bin_and_empty_curve(oracle):
    """One phase bin holds every point: the value is (sum w m)^2 / (2 sum w)
    at every trial period (rust/src/fpw.rs:46-63); an empty curve has no
    non-empty bin and scores 0."""
    rng = np.random.default_rng(4)
    t = lc.uniform_times(rng, 400, 100.0)
    m = lc.noisy(rng, lc.sinusoid(t, 2.2, amp=0.3, offset=15.0), 0.05)
    e = rng.uniform(0.05, 0.2, 400).astype(np.float32)
    P = lc.trial_periods(2.2, n=25)
    D = np.array([0.0, 1e-4], np.float32)
    got = oracle.fpw([t, np.zeros(0, np.float32)], [m, np.zeros(0, np.float32)], P, D, 1,
                     errs=[e, np.zeros(0, np.float32)])
    w = 1.0 / e.astype(np.float64) ** 2
    want = np.sum(w * m) ** 2 / (2.0 * np.sum(w))
    np.testing.assert_allclose(got[0], want, rtol=1e-5)
    assert np.all(got[0] == got[0, 0, 0])
    assert not got[1].any()


@pytest.mark.parametrize("case", [
    dict(period=5.0, n=800, noise=0.02, span=200.0, n_bins=20, errs=None),
    dict(period=3.0, n=600, noise=0.05, span=150.0, n_bins=15, errs="const"),
    dict(period=2.0, n=500, noise=0.03, span=100.0, n_bins=10, errs=None),
    dict(period=4.0, n=800, noise=None, span=200.0, n_bins=15, errs="var"),
])
def test_fpw_known_period(oracle, case):
    """Known-answer cases of the reference's CPU FPW tests
    (tests/test_cpu_standalone.py:412-465 and the variable-uncertainty case
    after it): the best period is the injected one to 5%."""
    rng = np.random.default_rng(42)
    t = lc.uniform_times(rng, case["n"], case["span"])
    if case["errs"] == "var":
        e = rng.uniform(0.01, 0.2, case["n"]).astype(np.float32)
        m = (lc.sinusoid(t, case["period"]) + rng.normal(0, 1, case["n"]) * e).astype(np.float32)
    else:
        m = lc.noisy(rng, lc.sinusoid(t, case["period"]), case["noise"])
        e = np.full(case["n"], 0.05, np.float32) if case["errs"] == "const" else None
    P = lc.trial_periods(case["period"], n=500)
    pg = oracle.fpw([t], [m], P, np.zeros(1, np.float32), case["n_bins"],
                    errs=None if e is None else [e])[0, :, 0]
    best = P[int(np.argmax(pg))]
    assert abs(best - case["period"]) / case["period"] < 0.05, best


def _bls_numpy(t, m, e, periods, pdts, n_bins, qmin, qmax):
    """BLS from numpy: the fold and f32 bin rule of rust/src/bls.rs:75-80, the
    weighted mean, bin sums, prefix sums and window search in float64."""
    t64 = t.astype(np.float64)
    w = (1.0 / (e.astype(np.float64) ** 2)) if e is not None else np.ones(len(t))
    yw = w * (m.astype(np.float64) - np.sum(w * m) / np.sum(w))
    lo = max(int(np.floor(np.float32(qmin) * np.float32(n_bins))), 1)
    hi = min(int(np.ceil(np.float32(qmax) * np.float32(n_bins))), n_bins - 1)
    out = np.zeros((len(periods), len(pdts)))
    for pi, P in enumerate(periods):
        for di, dt in enumerate(pdts):
            corr = np.float32(np.float32(dt) / np.float32(P)) / np.float32(2.0)
            r = (t64 - np.float64(corr) * t64 * t64) / np.float64(P)
            phase = np.abs(r - np.floor(r)).astype(np.float32)
            b = np.minimum((phase * np.float32(n_bins)).astype(np.int64), n_bins - 1)
            W = np.concatenate([[0.0], np.cumsum(np.bincount(b, weights=w, minlength=n_bins))])
            Y = np.concatenate([[0.0], np.cumsum(np.bincount(b, weights=yw, minlength=n_bins))])
            best = 0.0
            for nb in range(lo, hi + 1):
                for phi in range(n_bins):
                    end = phi + nb
                    if end <= n_bins:
                        rr, ss = W[end] - W[phi], Y[end] - Y[phi]
                    else:
                        rr = W[n_bins] - W[phi] + W[end - n_bins]
                        ss = Y[n_bins] - Y[phi] + Y[end - n_bins]
                    if 0 < rr / W[n_bins] < 1:
                        best = max(best, ss * ss / (rr * (W[n_bins] - rr)))
            out[pi, di] = best
    return out


def test_bls_matches_numpy_restatement(oracle):
    """The oracle's BLS (f32 sums in point order, as rust/src/bls.rs) is close
    to the same statistic in float64 (window sums difference-cancel, so the
    tolerance is looser than FPW's)."""
    rng = np.random.default_rng(5)
    t = lc.uniform_times(rng, 600, 200.0)
    m = lc.noisy(rng, lc.box_eclipse(t, 2.7, depth=0.3, duty=0.08) + 15.0, 0.02)
    e = rng.uniform(0.02, 0.2, 600).astype(np.float32)
    P = lc.trial_periods(2.7, n=40)
    D = np.array([0.0, 1e-4], np.float32)
    for errs, nb, q in ((None, 50, (0.01, 0.5)), ([e], 30, (0.02, 0.3)), ([e], 64, (0.0, 1.0))):
        got = oracle.bls([t], [m], P, D, nb, q[0], q[1], errs=errs)[0]
        want = _bls_numpy(t, m, None if errs is None else e, P, D, nb, *q)
        np.testing.assert_allclose(got, want, rtol=2e-3, atol=1e-6 * want.max())


@pytest.mark.parametrize("case", [
    dict(kind="eclipse", period=2.5, n=800, span=200.0, noise=0.02, qmax=0.3, errs=None),
    dict(kind="sine", period=5.0, n=800, span=200.0, noise=0.02, qmax=0.5, errs=None),
    dict(kind="eclipse", period=3.0, n=600, span=150.0, noise=0.05, qmax=0.3, errs=0.05),
    dict(kind="eclipse", period=2.0, n=500, span=100.0, noise=0.03, qmax=0.3, errs=None),
])
def test_bls_known_period(oracle, case):
    """Known-answer cases of the reference's CPU BLS tests
    (tests/test_cpu_standalone.py:555-640): the best period is the injected
    one, its half or its double, to 5%."""
    rng = np.random.default_rng(42)
    t = lc.uniform_times(rng, case["n"], case["span"])
    y = (lc.v_eclipse(t, case["period"]) if case["kind"] == "eclipse"
         else lc.sinusoid(t, case["period"]))
    m = lc.noisy(rng, y, case["noise"])
    e = None if case["errs"] is None else [np.full(case["n"], case["errs"], np.float32)]
    P = lc.trial_periods(case["period"], n=500)
    pg = oracle.bls([t], [m], P, np.zeros(1, np.float32), 50, 0.01, case["qmax"],
                    errs=e)[0, :, 0]
    best = float(P[int(np.argmax(pg))])
    assert any(abs(best - c) / c < 0.05 for c in (case["period"], case["period"] / 2,
                                                  case["period"] * 2)), best


def test_bls_degenerate_windows_score_zero(oracle):
    """BLS cells with no admissible window score 0 (rust/src/bls.rs:51-52,
    93-120): one bin (no width between 1 and n_bins - 1), qmin above qmax,
    an empty curve (no weight), and a single point (every window holds all
    of the weight or none of it)."""
    rng = np.random.default_rng(9)
    t = lc.uniform_times(rng, 300, 100.0)
    m = lc.noisy(rng, lc.box_eclipse(t, 3.1, depth=0.3) + 15.0, 0.02)
    P = lc.trial_periods(3.1, n=30)
    D = np.zeros(1, np.float32)
    assert not oracle.bls([t], [m], P, D, 1, 0.01, 0.5).any()
    assert not oracle.bls([t], [m], P, D, 50, 0.5, 0.1).any()
    e0 = np.zeros(0, np.float32)
    one_t, one_m = t[:1].copy(), m[:1].copy()
    out = oracle.bls([e0, one_t, t], [e0, one_m, m], P, D, 20, 0.05, 0.5)
    assert not out[0].any() and not out[1].any() and out[2].max() > 0
