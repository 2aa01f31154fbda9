"""Seeded synthetic light curves for the tests and the benchmark.

Signal shapes follow what the reference's tests exercise (sinusoids,
eclipsing binaries, sawtooth RR Lyrae-like curves, seasonal survey cadence:
tests/test_cpu_vs_cuda.py:54-96, tests/test_periodfind.py:890-938); the
generators themselves are written for this project.
"""

import numpy as np


def uniform_times(rng, n, t_span):
    return np.sort(rng.uniform(0.0, t_span, n)).astype(np.float32)


def seasonal_times(rng, n, baseline, season=125.25, year=365.25):
    """n times over `baseline` days, inside the first `season` days of each
    `year` (a 240-day annual gap for the defaults)."""
    n_years = int(np.ceil(baseline / year))
    yrs = rng.integers(0, n_years, n)
    t = yrs * year + rng.uniform(0.0, season, n)
    t = np.minimum(t, baseline)
    return np.sort(t).astype(np.float32)


def sinusoid(t, period, amp=1.0, phase=0.0, offset=1.0):
    return (offset + amp * np.sin(2.0 * np.pi * t.astype(np.float64) / period + phase))


def sawtooth(t, period, amp=1.0, phase=0.0):
    ph = np.mod(t.astype(np.float64) / period + phase, 1.0)
    return amp * (2.0 * ph - 1.0)


def box_eclipse(t, period, depth=0.5, duty=0.05, phase=0.0):
    ph = np.mod(t.astype(np.float64) / period + phase, 1.0)
    return np.where(ph < duty, -depth, 0.0)


def v_eclipse(t, period, depth=0.5, width=0.1):
    ph = np.mod(t.astype(np.float64) / period, 1.0)
    d = np.minimum(ph, 1.0 - ph)
    return np.where(d < width / 2, 1.0 - depth * (1.0 - d / (width / 2)), 1.0)


def rr_lyrae(t, period, amp=0.8, rise=0.2):
    ph = np.mod(t.astype(np.float64) / period, 1.0)
    return np.where(ph < rise, amp * ph / rise, amp * (1.0 - (ph - rise) / (1.0 - rise)))


def noisy(rng, y, sigma):
    return (y + rng.normal(0.0, sigma, len(y))).astype(np.float32)


def sine_curve(period, n=500, t_span=100.0, noise=0.05, seed=42, amp=1.0):
    rng = np.random.default_rng(seed)
    t = uniform_times(rng, n, t_span)
    return t, noisy(rng, sinusoid(t, period, amp=amp, offset=amp), noise)


def eclipse_curve(period, n=600, t_span=200.0, noise=0.02, seed=42):
    rng = np.random.default_rng(seed)
    t = uniform_times(rng, n, t_span)
    return t, noisy(rng, v_eclipse(t, period), noise)


def rrl_curve(period, n=600, t_span=50.0, noise=0.02, seed=42):
    rng = np.random.default_rng(seed)
    t = uniform_times(rng, n, t_span)
    return t, noisy(rng, rr_lyrae(t, period), noise)


def trial_periods(true_period, n=200, margin=0.5):
    lo = max(true_period * (1.0 - margin), 0.01)
    return np.linspace(lo, true_period * (1.0 + margin), n, dtype=np.float32)


def normalize(m):
    """The reference's normalize=True preparation (periodfind/_utils.py:39-45)."""
    lo, hi = np.min(m), np.max(m)
    return ((m - lo) / (hi - lo)) * 0.999 + 5e-4


def center(m):
    return m - np.mean(m)


def mixed_signal_batch(n_curves, n_points, seed, t_span=2000.0):
    """Curves shaped like the 1000 x 4096 benchmark batch: half sinusoids,
    a quarter sawtooth, a quarter box eclipses (depth 0.5, duty 0.05),
    N(0, 0.05^2) noise, periods log-uniform in [0.1, 100] days."""
    rng = np.random.default_rng(seed)
    times, mags = [], []
    for i in range(n_curves):
        t = uniform_times(rng, n_points, t_span)
        p = float(np.exp(rng.uniform(np.log(0.1), np.log(100.0))))
        ph = rng.uniform(0, 1)
        kind = i % 4
        if kind < 2:
            y = sinusoid(t, p, amp=rng.uniform(0.1, 0.5), phase=2 * np.pi * ph, offset=0.0)
        elif kind == 2:
            y = sawtooth(t, p, amp=rng.uniform(0.1, 0.5), phase=ph)
        else:
            y = box_eclipse(t, p, 0.5, 0.05, ph)
        times.append(t)
        mags.append(noisy(rng, y, 0.05))
    return times, mags


def ls_study_curves(n_curves, seed, lengths=None, baseline=3000.0):
    """Lomb-Scargle study curves: lengths log-uniform in [64, 16384] unless
    given; seasonal cadence over `baseline` days with a 240-day annual gap;
    15 + A sin(2 pi f t) + N(0, sigma^2), A ~ U[0.01, 0.5], sigma ~ U[0.01,
    0.1], f ~ U[0.01, 20] per day.  Returns (times, mags, freqs, sigmas)
    with float32 times / mags and the magnitudes centred."""
    rng = np.random.default_rng(seed)
    if lengths is None:
        lengths = np.exp(rng.uniform(np.log(64), np.log(16384), n_curves)).astype(np.int64)
    ts, ms, fs, ss = [], [], [], []
    for n in lengths:
        t = seasonal_times(rng, int(n), baseline)
        a, s, f = rng.uniform(0.01, 0.5), rng.uniform(0.01, 0.1), rng.uniform(0.01, 20.0)
        m = 15.0 + a * np.sin(2 * np.pi * f * t.astype(np.float64) + rng.uniform(0, 2 * np.pi))
        m = (m + rng.normal(0.0, s, len(t))).astype(np.float32)
        ts.append(t)
        ms.append(center(m))
        fs.append(f)
        ss.append(s)
    return ts, ms, np.array(fs), np.array(ss)
