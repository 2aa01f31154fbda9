"""Bin occupancies count for count, then the statistics on identical bins.

The CE and AOV periodograms are functions of their bins.  Here the raw bin
counts of the plain and chosen kernels (pf_bin_counts) are compared, cell
by cell and bin by bin, with

  - semantics='cuda': the reference CUDA build's own bins, from its
    FoldAndBin step run on the GPU (ConditionalEntropy::DeviceFoldAndBin,
    periodfind/cuda/ce.cu:262-290; AOV::DeviceFoldAndBin, aov.cu:265-299);
  - semantics='cpu': the oracle's bins (the Rust path's fold and bin rule,
    rust/src/fold.rs:13-26, ce.rs:78-89, aov.rs:172-180),

on the lengths the reference's tests exercise at block boundaries (1, 2,
5, 31-33, 255-257, 4096, 4097), seasonal MJD-like baselines (t ~ 58000 d)
and period derivatives.  Tolerance: none (array_equal).

With the bins pinned, the AOV statistic is checked against an FP64
statistic on the same bins (the oracle's, on cells where its bins equal the
reference's):
  - chosen form (exact fixed-point bin sums, FP64 statistic): within 1e-5
    relative at every cell;
  - plain form and the reference: f32 sums whose rounding depends on the
    summation order (the plain form adds in point order, the reference with
    shared float atomics in no fixed order).  The plain form's error against
    the FP64 statistic is that of the f32 statistic summed in point order
    (the oracle, the Rust path's order): at most 1.25 times it at the
    median and the 99th percentile over cells.  The reference's own error is
    printed beside it.
"""

import numpy as np
import pytest

import lightcurves as lc

pytestmark = pytest.mark.gpu

EDGE_LENGTHS = (1, 2, 5, 31, 32, 33, 255, 256, 257, 4096, 4097)
PERIODS = np.exp(np.linspace(np.log(0.1), np.log(50.0), 150)).astype(np.float32)
PDTS = np.array([0.0, 1e-6, -2e-5], np.float32)


@pytest.fixture(scope="module")
def gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from periodfind_b200 import gpu as g

    return g


def _ref_or_skip(oracle):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/libpfref.so not built (needs the reference checkout)")


def _curves(seed, raw=False):
    """Edge-length curves over 300 days and two MJD-like seasonal curves;
    magnitudes normalised into (0, 1) unless raw."""
    rng = np.random.default_rng(seed)
    ts, ms = [], []
    for n in EDGE_LENGTHS:
        t = lc.uniform_times(rng, n, 300.0)
        ts.append(t)
        ms.append(lc.noisy(rng, 15.0 + 0.3 * np.sin(2 * np.pi * t / rng.uniform(1, 5)), 0.05))
    for n in (500, 2000):
        t = (58000.0 + lc.seasonal_times(rng, n, 3000.0)).astype(np.float32)
        ts.append(t)
        ms.append(lc.noisy(rng, 15.0 + lc.box_eclipse(t, rng.uniform(0.5, 3.0)), 0.02))
    if not raw:
        ms = [lc.normalize(m) if len(m) > 1 else np.full(1, 0.5, np.float32) for m in ms]
    return ts, ms


@pytest.mark.parametrize("overlap", [(1, 1), (2, 3)])
def test_ce_bins_equal_reference_cuda(gpu, oracle, overlap):
    _ref_or_skip(oracle)
    po, mo = overlap
    ts, ms = _curves(21)
    for mode in ("plain", "chosen"):
        ce = gpu.ConditionalEntropy(10, 10, po, mo, mode=mode)
        _, got = ce.bin_counts(ts, ms, PERIODS, PDTS)
        for c, (t, m) in enumerate(zip(ts, ms)):
            want = oracle.ref_fold_and_bin("ce", t, m, PERIODS, PDTS, 10, 10, po, mo)
            np.testing.assert_array_equal(got[c], want, err_msg=f"{mode} curve {c} ({len(t)})")


@pytest.mark.parametrize("overlap", [1, 2])
def test_aov_bins_equal_reference_cuda(gpu, oracle, overlap):
    _ref_or_skip(oracle)
    ts, ms = _curves(22, raw=True)
    for mode in ("plain", "chosen"):
        aov = gpu.AOV(15, overlap, mode=mode)
        _, got = aov.bin_counts(ts, ms, PERIODS, PDTS)
        for c, (t, m) in enumerate(zip(ts, ms)):
            want, _, _ = oracle.ref_fold_and_bin("aov", t, m, PERIODS, PDTS, 15, po=overlap)
            np.testing.assert_array_equal(got[c], want, err_msg=f"{mode} curve {c} ({len(t)})")


def test_bins_equal_oracle_cpu_semantics(gpu, oracle):
    """semantics='cpu' against the Rust path's bins (the oracle), CE and AOV,
    both forms, every cell of a subset of the curves."""
    ts, ms = _curves(23)
    pick = [0, 2, 4, 7, 8, 10, 11, 12]
    ts, ms = [ts[i] for i in pick], [ms[i] for i in pick]
    per, pdt = PERIODS[::5], PDTS
    for mode in ("plain", "chosen"):
        _, ce = gpu.ConditionalEntropy(10, 10, mode=mode, semantics="cpu").bin_counts(
            ts, ms, per, pdt)
        _, aov = gpu.AOV(15, mode=mode, semantics="cpu").bin_counts(ts, ms, per, pdt)
        for c, (t, m) in enumerate(zip(ts, ms)):
            for i, P in enumerate(per):
                for k, D in enumerate(pdt):
                    _, w = oracle.ce_counts(t, m, P, D, 10, 10)
                    np.testing.assert_array_equal(ce[c, i, k], w.ravel(), err_msg=f"CE {mode}")
                    _, w = oracle.aov_counts(t, m, P, D, 15)
                    np.testing.assert_array_equal(aov[c, i, k], w, err_msg=f"AOV {mode}")


@pytest.mark.parametrize("raw", [False, True], ids=["normalised", "raw-15pm0.3"])
def test_aov_statistic_on_identical_bins(gpu, oracle, raw):
    """The AOV statistic where the bins are pinned equal to the reference's."""
    _ref_or_skip(oracle)
    ts, ms = _curves(24, raw=raw)
    keep = [c for c, t in enumerate(ts) if len(t) >= 31]  # AOV needs n > n_bins
    ts, ms = [ts[c] for c in keep], [ms[c] for c in keep]
    ref = oracle.ref_cuda("aov", ts, ms, PERIODS, PDTS, n_phase=15)
    plain, counts = gpu.AOV(15, mode="plain").bin_counts(ts, ms, PERIODS, PDTS)
    chosen, counts_c = gpu.AOV(15, mode="chosen").bin_counts(ts, ms, PERIODS, PDTS)
    np.testing.assert_array_equal(counts, counts_c)
    truth = oracle.aov_f64(ts, ms, PERIODS, PDTS, 15, fused_tcorr=True)
    # Cells where the oracle's bins (IEEE f32 divide in the bin rule) equal
    # the reference's (fast-math divide): the FP64 statistic is then the
    # exact value of the reference's binning.
    same = np.ones(truth.shape, bool)
    for c, (t, m) in enumerate(zip(ts, ms)):
        want, _, _ = oracle.ref_fold_and_bin("aov", t, m, PERIODS, PDTS, 15)
        np.testing.assert_array_equal(counts[c], want)
        for i, P in enumerate(PERIODS):
            for k, D in enumerate(PDTS):
                _, w = oracle.aov_counts(t, m, P, D, 15, fused_tcorr=True)
                same[c, i, k] = np.array_equal(w, want[i, k])
    # The two bin rules differ only for a point within the fast-math
    # divide's 2 ulp of a bin edge; a 4096-point curve has such a point in
    # a few percent of its cells.
    assert same.mean() > 0.9
    scale = np.abs(truth).max(axis=(1, 2), keepdims=True)
    rel = lambda x: (np.abs(x - truth) / (np.abs(truth) + 1e-6 * scale))[same]
    seq = oracle.aov(ts, ms, PERIODS, PDTS, 15, fused_tcorr=True)
    e_chosen, e_plain, e_ref, e_seq = rel(chosen), rel(plain), rel(ref), rel(seq)
    print(f"\nAOV vs FP64 on identical bins ({'raw' if raw else 'normalised'}): "
          f"chosen max {e_chosen.max():.2e}; plain max {e_plain.max():.2e} median "
          f"{np.median(e_plain):.2e}; reference max {e_ref.max():.2e} median "
          f"{np.median(e_ref):.2e}; plain within 1e-5 of the reference at "
          f"{np.mean(np.abs(plain - ref)[same] <= 1e-5 * np.abs(ref)[same] + 1e-6):.4f}")
    assert e_chosen.max() <= 1e-5
    for q in (0.5, 0.99):
        assert np.quantile(e_plain, q) <= 1.25 * np.quantile(e_seq, q) + 1e-7


def test_ce_statistic_on_identical_bins(gpu, oracle):
    """CE: with the bins equal to the reference's, the plain form's value
    differs from the reference CUDA build only in the order of its float
    additions over phase rows (ce.cu:243-253): within 1e-5 relative; the
    chosen form's divide-free statistic also within 1e-5."""
    _ref_or_skip(oracle)
    ts, ms = _curves(25)
    ref = oracle.ref_cuda("ce", ts, ms, PERIODS, PDTS, n_phase=10, n_mag=10)
    for mode in ("plain", "chosen"):
        got, _ = gpu.ConditionalEntropy(10, 10, mode=mode).bin_counts(ts, ms, PERIODS, PDTS)
        np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-7)
