"""Lomb-Scargle on a uniform frequency grid (pf_ls_fgrid): the MUFU sincos
form and the angle-addition recurrence along the grid, against the FP64
oracle evaluated at the same exact frequencies, on the precision-study
cadence (seasonal, 3000 days, up to 6e4 cycles at 20 / day).

Bounds (of each curve's largest FP64 power):
  sincos form       |err| <= 2e-5, the bound of the split-precision fold on
                    a period grid (tests/test_gpu_precision.py)
  recurrence form   |err| <= 4e-5 (up to 7 rotations in f32 after the
                    first MUFU pair), and the same grid argmax as FP64
  exact fold        |err| <= 2e-5
The tuner's choice is reported per length class, and both forms agree on
tiny and empty curves.
"""

import numpy as np
import pytest

import lightcurves as lc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from periodfind_b200 import gpu as g

    return g


def _grid(n_freq=6000, f_min=0.01, f_max=20.0):
    df = (f_max - f_min) / (n_freq - 1)
    return f_min, df, n_freq


def test_frequency_grid_vs_fp64(gpu, oracle):
    lengths = [40, 64, 300, 1500, 4000, 9000]
    ts, ms, fs, _ = lc.ls_study_curves(len(lengths), seed=31, lengths=lengths)
    f_min, df, n = _grid()
    freqs = f_min + np.arange(n) * df
    ref = oracle.ls_f64(ts, ms, 1.0 / freqs, [0.0])[:, :, 0]
    scale = ref.max(axis=1, keepdims=True)
    ls = gpu.LombScargle()
    errs = {}
    for trig, bound in (("sincos", 2e-5), ("recurrence", 4e-5)):
        pg = ls.periodograms_frequency_grid(ts, ms, f_min, df, n, trig=trig, center=False)
        err = np.abs(pg - ref) / scale
        errs[trig] = float(err.max())
        assert err.max() <= bound, (trig, err.max(axis=1))
        assert np.array_equal(np.argmax(pg, axis=1), np.argmax(ref, axis=1)), trig
    exact = gpu.LombScargle(fold="exact").periodograms_frequency_grid(ts, ms, f_min, df, n,
                                                                      center=False)
    errs["exact"] = float((np.abs(exact - ref) / scale).max())
    assert errs["exact"] <= 2e-5
    tuned = ls.periodograms_frequency_grid(ts, ms, f_min, df, n, center=False)
    errs["tuned"] = float((np.abs(tuned - ref) / scale).max())
    assert errs["tuned"] <= 4e-5
    print("\nfrequency-grid LS power error vs FP64 (of each curve's peak):", errs)


def test_tuner_reports_trig_choice(gpu):
    from periodfind_b200 import _native as nat

    lengths = [30, 100, 500, 2000, 5000] * 4
    ts, ms, _, _ = lc.ls_study_curves(len(lengths), seed=32, lengths=lengths)
    f_min, df, n = _grid(3000)
    gpu.LombScargle().periodograms_frequency_grid(ts, ms, f_min, df, n)
    rep = [ln for ln in nat.default_context(0).tuning_report().splitlines()
           if "fold-split-fgrid " in ln]
    print("\n" + "\n".join(rep))
    assert len(rep) == 5 and all("trig=" in ln for ln in rep)


def test_tiny_and_empty_curves(gpu):
    rng = np.random.default_rng(33)
    ts, ms = [], []
    for n in (0, 1, 2, 3, 7, 513):
        t = lc.seasonal_times(rng, n, 3000.0)
        ts.append(t)
        ms.append((rng.normal(0, 1, n)).astype(np.float32))
    f_min, df, n = _grid(1100, 0.5, 3.0)
    ls = gpu.LombScargle()
    a = ls.periodograms_frequency_grid(ts, ms, f_min, df, n, trig="sincos", center=False)
    b = ls.periodograms_frequency_grid(ts, ms, f_min, df, n, trig="recurrence", center=False)
    # The 513-point curve: the two forms agree to the recurrence's bound.
    scale = np.abs(a[-1]).max()
    assert np.all(np.abs(a[-1] - b[-1]) <= 4e-5 * scale)
    # An empty curve gives the sincos form's value in both (0 / 0 in the
    # reference CUDA build's arithmetic); curves of a handful of points have
    # a nearly singular normal matrix and are only run.
    np.testing.assert_array_equal(np.isnan(a[0]), np.isnan(b[0]))


def test_grid_arguments_checked(gpu):
    from periodfind_b200 import _native as nat

    t = np.linspace(0, 10, 20).astype(np.float32)
    with pytest.raises(ValueError):
        gpu.LombScargle(mode="plain").periodograms_frequency_grid([t], [t], 0.1, 0.01, 10)
    with pytest.raises(nat.PeriodfindError):
        gpu.LombScargle().periodograms_frequency_grid([t], [t], float("nan"), 0.01, 10)
