"""Seeded synthetic light curves for the tests and the benchmark (bench.py).

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


def ragged_batch(n_curves, seed, baseline=2500.0):
    """The mixed ragged batch: lengths lognormal (median 300, sigma 0.8)
    rounded and clipped to [20, 2000]; seasonal cadence over `baseline` days
    (125.25-day seasons, a 240-day annual gap); a third sinusoids
    (amplitude 0.3), a third box eclipses (depth 0.5, duty 0.05), a third
    pure noise, periods log-uniform in [0.05, 500] d; noise sigma U[0.02,
    0.1] per curve; magnitudes around 15.  Returns CSR (times float32,
    mags float32, offsets int64), curve c = [off[c], off[c+1])."""
    rng = np.random.default_rng(seed)
    lens = np.clip(np.round(rng.lognormal(np.log(300.0), 0.8, n_curves)), 20, 2000).astype(np.int64)
    cid = np.repeat(np.arange(n_curves), lens)
    n_years = int(np.ceil(baseline / 365.25))
    t = rng.integers(0, n_years, cid.size) * 365.25 + rng.uniform(0.0, 125.25, cid.size)
    t = np.minimum(t, baseline)
    order = np.lexsort((t, cid))
    t = t[order].astype(np.float32)
    period = np.exp(rng.uniform(np.log(0.05), np.log(500.0), n_curves))[cid]
    phase = rng.uniform(0, 1, n_curves)[cid]
    kind = (np.arange(n_curves) % 3)[cid]
    sigma = rng.uniform(0.02, 0.1, n_curves)[cid]
    ph = np.mod(t / period + phase, 1.0)
    y = np.where(kind == 0, 0.3 * np.sin(2 * np.pi * ph),
                 np.where(kind == 1, np.where(ph < 0.05, -0.5, 0.0), 0.0))
    m = (15.0 + y + rng.normal(0.0, 1.0, cid.size) * sigma).astype(np.float32)
    off = np.zeros(n_curves + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    return t, m, off


def seasonal_ls_batch(lengths, seed, baseline=3000.0):
    """LS study curves as CSR: seasonal cadence over `baseline` days
    (240-day annual gap), 15 + A sin(2 pi f t) + N(0, sigma^2) with A ~
    U[0.01, 0.5], sigma ~ U[0.01, 0.1], f ~ U[0.01, 20] / day; magnitudes
    centred.  Returns (times float32, mags float32, offsets int64)."""
    rng = np.random.default_rng(seed)
    lengths = np.asarray(lengths, np.int64)
    n_curves = len(lengths)
    cid = np.repeat(np.arange(n_curves), lengths)
    n_years = int(np.ceil(baseline / 365.25))
    t = rng.integers(0, n_years, cid.size) * 365.25 + rng.uniform(0.0, 125.25, cid.size)
    t = np.minimum(t, baseline)
    t = t[np.lexsort((t, cid))].astype(np.float32)
    amp = rng.uniform(0.01, 0.5, n_curves)[cid]
    sig = rng.uniform(0.01, 0.1, n_curves)[cid]
    f = rng.uniform(0.01, 20.0, n_curves)[cid]
    ph = rng.uniform(0, 2 * np.pi, n_curves)[cid]
    m = 15.0 + amp * np.sin(2 * np.pi * f * t.astype(np.float64) + ph)
    m = m + rng.normal(0.0, 1.0, cid.size) * sig
    off = np.zeros(n_curves + 1, np.int64)
    np.cumsum(lengths, out=off[1:])
    mean = np.add.reduceat(m, off[:-1]) / lengths
    return t, (m - mean[cid]).astype(np.float32), off


def split_csr(flat, off):
    """The curves of a CSR array as a list of views (no copies)."""
    return np.split(flat, off[1:-1])
