"""BLS (box least squares) on the device against the oracle (the Rust path's
arithmetic) and the reference's own CUDA build, and the drop-in class's
behaviour (periodfind/bls.pyx:36-181, periodfind/cpu/__init__.py:525-640;
the reference's tests/test_cpu_standalone.py:555-640)."""

import numpy as np
import pytest

from periodfind_b200 import Periodogram, Statistics
import lightcurves as lc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from periodfind_b200 import gpu as g

    return g


@pytest.fixture(scope="module")
def oracle():
    from oracle import oracle as O

    return O


def _batch(seed=4, lengths=(0, 1, 2, 7, 33, 255, 257, 1023, 2500)):
    rng = np.random.default_rng(seed)
    ts, ms, es = [], [], []
    for n in lengths:
        t = lc.uniform_times(rng, n, 400.0)
        ts.append(t)
        ms.append(lc.noisy(rng, 15.0 + lc.box_eclipse(t, float(rng.uniform(0.5, 10)),
                                                      depth=0.3, duty=0.05), 0.05))
        es.append(rng.uniform(0.02, 0.3, n).astype(np.float32))
    return ts, ms, es


def _grid(n=300, pdts=(0.0, 1e-4)):
    P = np.exp(np.linspace(np.log(0.3), np.log(30.0), n)).astype(np.float32)
    return P, np.array(pdts, np.float32)


@pytest.mark.parametrize("mode", ["plain", "chosen"])
@pytest.mark.parametrize("cfg", [(50, 0.01, 0.5), (20, 0.05, 0.2), (7, 0.0, 1.0), (100, 0.01, 0.1)])
def test_bls_cpu_semantics_equals_oracle(gpu, oracle, mode, cfg):
    """semantics='cpu': the Rust path's fold, bin rule, point-order f32 sums,
    prefix sums and window search, so the values are the oracle's bit for
    bit (ragged lengths 0 to 2500, per-point uncertainties, two period
    derivatives).  The IEEE r / W is exactly 1 for a window holding all the
    weight, so no cell is infinite here."""
    nb, qmin, qmax = cfg
    ts, ms, es = _batch()
    P, D = _grid()
    obj = gpu.BoxLeastSquares(nb, qmin, qmax, mode=mode, semantics="cpu")
    got = obj.periodograms(ts, ms, P, D, errs=es)
    assert np.isfinite(got).all()
    np.testing.assert_array_equal(got, oracle.bls(ts, ms, P, D, nb, qmin, qmax, errs=es))
    np.testing.assert_array_equal(obj.periodograms(ts, ms, P, D),
                                  oracle.bls(ts, ms, P, D, nb, qmin, qmax))


@pytest.mark.parametrize("semantics", ["cuda", "cpu"])
def test_bls_chosen_equals_plain_long_baselines(gpu, semantics):
    """The chosen form's fast bins give the plain form's bins, so the values
    are equal bit for bit, also at MJD-like times with short periods."""
    rng = np.random.default_rng(17)
    ts, ms, es = [], [], []
    for n in (300, 2000, 4097):
        t = np.sort(rng.uniform(58000.0, 60000.0, n)).astype(np.float32)
        ts.append(t)
        ms.append(lc.noisy(rng, lc.box_eclipse(t, 0.0371, depth=0.3, duty=0.05), 0.05))
        es.append(rng.uniform(0.02, 0.2, n).astype(np.float32))
    P = np.exp(np.linspace(np.log(0.01), np.log(0.1), 500)).astype(np.float32)
    D = np.array([0.0, 1e-7], np.float32)
    a = gpu.BoxLeastSquares(mode="plain", semantics=semantics).periodograms(ts, ms, P, D, errs=es)
    b = gpu.BoxLeastSquares(mode="chosen", semantics=semantics).periodograms(ts, ms, P, D,
                                                                              errs=es)
    np.testing.assert_array_equal(a, b)


def test_bls_cuda_semantics_vs_reference_cuda(gpu, oracle):
    """semantics='cuda' against the reference's CUDA build run on this GPU:
    the same fold, bin rule and window search; the reference adds a bin's
    weights in no fixed order (float atomics or warp reductions) and window
    sums are differences of prefix sums, so the values agree to f32 rounding
    amplified by that cancellation.  Both score inf where a window holds all
    the weight (the fast-math r / W falls just below 1 when r == W), which
    the 5-point curve meets: those cells must coincide."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/libpfref.so not built (needs the reference checkout)")
    ts, ms, es = _batch(seed=6, lengths=(5, 64, 300, 1000, 2048, 5000, 9000))
    P, D = _grid(200)
    for nb, qmin, qmax in ((50, 0.01, 0.5), (32, 0.05, 0.2)):
        want = oracle.ref_cuda("bls", ts, ms, P, D, n_bins=nb, qmin=qmin, qmax=qmax, errs=es)
        got = gpu.BoxLeastSquares(nb, qmin, qmax).periodograms(ts, ms, P, D, errs=es)
        np.testing.assert_array_equal(np.isinf(got), np.isinf(want))
        fin = np.isfinite(want)
        assert fin.sum() > 0.9 * want.size
        np.testing.assert_allclose(got[fin], want[fin], rtol=2e-3,
                                   atol=1e-5 * np.abs(want[fin]).max())


def test_bls_outputs_and_errors(gpu, oracle):
    """The reference's CPU BLS contract: Statistics and Periodogram outputs
    (maximum is best), n_stats > 1, the errs checks, and 'peaks' equal to
    the oracle's peak search on the same periodogram."""
    t, m = lc.eclipse_curve(2.5, n=500)
    P = np.linspace(1.0, 10.0, 100, dtype=np.float32)
    D2 = np.array([0.0, 0.001], np.float32)
    obj = gpu.BoxLeastSquares()
    r = obj.calc([t], [m], P, np.zeros(1, np.float32), output="stats")
    assert isinstance(r[0], Statistics) and r[0].significance > 0
    pg = obj.calc([t], [m], P, D2, output="periodogram")[0]
    assert isinstance(pg, Periodogram) and pg.data.shape == (100, 2) and pg.use_max is True
    assert len(obj.calc([t], [m], P, np.zeros(1, np.float32), n_stats=5)[0]) == 5
    with pytest.raises(ValueError):
        obj.calc([t, t], [m, m], P, D2, errs=[np.ones(len(t), np.float32)])
    with pytest.raises(TypeError, match="expected float32"):
        obj.calc([t], [m], P, D2, errs=[np.ones(len(t), np.float64)])
    with pytest.raises(RuntimeError):
        gpu.BoxLeastSquares(n_bins=0).calc([t], [m], P, D2)
    ts, ms, es = _batch(seed=7)
    Pg, Dg = _grid(1500, pdts=(0.0, 2e-5))
    data = obj.periodograms(ts, ms, Pg, Dg, errs=es)
    for n_peaks, md in ((8, 1), (32, 5)):
        idx, val = obj.peaks(ts, ms, Pg, Dg, n_peaks, md, errs=es)
        oi, ov = oracle.find_top_peaks_batched(data, n_peaks, md, True)
        np.testing.assert_array_equal(idx, oi)
        np.testing.assert_array_equal(val, ov)
    assert len(obj.calc(ts, ms, Pg, Dg, errs=es, output="peaks", n_peaks=8)) == len(ts)


@pytest.mark.parametrize("errs", [None, 0.05])
def test_bls_detects_eclipsing_binary(gpu, errs):
    """Known-answer detection on the device (the reference's
    tests/test_cpu_standalone.py:576-620): the injected period, its half or
    its double, to 5%."""
    rng = np.random.default_rng(42)
    t = lc.uniform_times(rng, 800, 200.0)
    m = lc.noisy(rng, lc.v_eclipse(t, 2.5), 0.02)
    e = None if errs is None else [np.full(800, errs, np.float32)]
    P = lc.trial_periods(2.5, n=500)
    r = gpu.BoxLeastSquares(50, 0.01, 0.3).calc([t], [m], P, np.zeros(1, np.float32), errs=e)
    best = float(r[0].params[0])
    assert any(abs(best - c) / c < 0.05 for c in (2.5, 1.25, 5.0)), best


@pytest.mark.parametrize("mode", ["plain", "chosen"])
def test_bls_degenerate_windows_score_zero(gpu, oracle, mode):
    """No admissible window: one bin, qmin above qmax, an empty curve, a
    single point.  In the Rust path's arithmetic those cells are 0, as the
    oracle's (rust/src/bls.rs:51-52, 93-120)."""
    rng = np.random.default_rng(9)
    t = lc.uniform_times(rng, 300, 100.0)
    m = lc.noisy(rng, lc.box_eclipse(t, 3.1, depth=0.3) + 15.0, 0.02)
    P = lc.trial_periods(3.1, n=30)
    D = np.array([0.0, 1e-4], np.float32)
    e0 = np.zeros(0, np.float32)
    ts, ms = [e0, t[:1].copy(), t], [e0, m[:1].copy(), m]
    for nb, qmin, qmax in ((1, 0.01, 0.5), (50, 0.5, 0.1), (20, 0.05, 0.5)):
        got = gpu.BoxLeastSquares(nb, qmin, qmax, mode=mode, semantics="cpu").periodograms(
            ts, ms, P, D)
        want = oracle.bls(ts, ms, P, D, nb, qmin, qmax)
        np.testing.assert_array_equal(got, want)
        assert not got[0].any() and not got[1].any()
