"""FPW on the device against the oracle (the Rust path's arithmetic) and the
reference's own CUDA build, and the drop-in class's behaviour
(periodfind/fpw.pyx:29-177, periodfind/cpu/__init__.py:400-521; the
reference's tests/test_cpu_standalone.py:393-540)."""

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


def _batch(seed=4, lengths=(0, 1, 2, 7, 31, 32, 33, 255, 256, 257, 1023, 1025, 2500)):
    rng = np.random.default_rng(seed)
    ts, ms, es = [], [], []
    for n in lengths:
        t = lc.uniform_times(rng, n, 400.0)
        ts.append(t)
        ms.append(lc.noisy(rng, lc.sinusoid(t, float(rng.uniform(0.5, 10)), amp=0.3,
                                             offset=15.0), 0.05))
        es.append(rng.uniform(0.02, 0.3, n).astype(np.float32))
    return ts, ms, es


def _grid(n=700, pdts=(0.0, 1e-4, -3e-4)):
    P = np.exp(np.linspace(np.log(0.2), np.log(50.0), n)).astype(np.float32)
    return P, np.array(pdts, np.float32)


@pytest.mark.parametrize("mode", ["plain", "chosen"])
@pytest.mark.parametrize("n_bins", [10, 20, 7, 100])
def test_fpw_cpu_semantics_equals_oracle(gpu, oracle, mode, n_bins):
    """semantics='cpu': the Rust path's fold, bin rule and point-order f32
    sums, so the values are the oracle's bit for bit (ragged lengths 0 to
    2500, per-point uncertainties, three period derivatives)."""
    ts, ms, es = _batch()
    P, D = _grid()
    obj = gpu.FPW(n_bins, mode=mode, semantics="cpu")
    np.testing.assert_array_equal(obj.periodograms(ts, ms, P, D, errs=es),
                                  oracle.fpw(ts, ms, P, D, n_bins, errs=es))
    np.testing.assert_array_equal(obj.periodograms(ts, ms, P, D),
                                  oracle.fpw(ts, ms, P, D, n_bins))


def test_fpw_chosen_equals_plain(gpu):
    """The chosen form's fast bins (the reference sequence within the guard
    of a bin edge) are the plain form's bins, so its values equal the plain
    form's bit for bit."""
    ts, ms, es = _batch(seed=5)
    P, D = _grid(900)
    a = gpu.FPW(15, mode="plain").periodograms(ts, ms, P, D, errs=es)
    b = gpu.FPW(15, mode="chosen").periodograms(ts, ms, P, D, errs=es)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("n_bins", [10, 20])
def test_fpw_cuda_semantics_vs_reference_cuda(gpu, oracle, n_bins):
    """semantics='cuda' against the reference's CUDA build run on this GPU:
    the same fold and bin rule; the reference adds a bin's weights with float
    atomics or warp reductions in no fixed order, so the values agree to f32
    rounding of the sums, not bit for bit."""
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/libpfref.so not built (needs the reference checkout)")
    ts, ms, es = _batch(seed=6, lengths=(5, 64, 300, 1000, 2048, 3000, 5000))
    P, D = _grid(400, pdts=(0.0, 1e-4))
    want = oracle.ref_cuda("fpw", ts, ms, P, D, n_bins=n_bins, errs=es)
    got = gpu.FPW(n_bins).periodograms(ts, ms, P, D, errs=es)
    np.testing.assert_allclose(got, want, rtol=2e-5, atol=1e-6 * np.abs(want).max())


def test_fpw_outputs_and_errors(gpu, oracle):
    """The reference's CPU FPW contract: Statistics and Periodogram outputs
    (maximum is best), n_stats > 1, the errs checks, and 'peaks' equal to
    the oracle's peak search on the same periodogram."""
    t, m = lc.sine_curve(3.0, n=500)
    P = np.linspace(1.0, 10.0, 100, dtype=np.float32)
    D2 = np.array([0.0, 0.001], np.float32)
    obj = gpu.FPW(n_bins=10)
    r = obj.calc([t], [m], P, np.zeros(1, np.float32), output="stats")
    assert isinstance(r[0], Statistics) and r[0].significance > 0
    pg = obj.calc([t], [m], P, D2, output="periodogram")[0]
    assert isinstance(pg, Periodogram) and pg.data.shape == (100, 2) and pg.use_max is True
    assert len(obj.calc([t], [m], P, np.zeros(1, np.float32), n_stats=5)[0]) == 5
    with pytest.raises(ValueError):
        obj.calc([t, t], [m, m], P, D2, errs=[np.ones(len(t), np.float32)])
    with pytest.raises(ValueError):
        obj.calc([t], [m], P, D2, errs=[np.ones(len(t) - 1, np.float32)])
    with pytest.raises(TypeError, match="expected float32"):
        obj.calc([t], [m], P, D2, errs=[np.ones(len(t), np.float64)])
    with pytest.raises(RuntimeError):
        gpu.FPW(n_bins=200).calc([t], [m], P, D2)
    ts, ms, es = _batch(seed=7)
    Pg, Dg = _grid(1500, pdts=(0.0, 2e-5))
    data = obj.periodograms(ts, ms, Pg, Dg, errs=es)
    for n_peaks, md in ((8, 1), (32, 5)):
        idx, val = obj.peaks(ts, ms, Pg, Dg, n_peaks, md, errs=es)
        oi, ov = oracle.find_top_peaks_batched(data, n_peaks, md, True)
        np.testing.assert_array_equal(idx, oi)
        np.testing.assert_array_equal(val, ov)
    res = obj.calc(ts, ms, Pg, Dg, errs=es, output="peaks", n_peaks=8)
    assert len(res) == len(ts)


@pytest.mark.parametrize("errs", [None, "const", "var"])
def test_fpw_detects_known_period(gpu, errs):
    """Known-answer detection on the device, with no, constant and variable
    uncertainties (the reference's tests/test_cpu_standalone.py:412-540)."""
    rng = np.random.default_rng(42)
    t = lc.uniform_times(rng, 800, 200.0)
    if errs == "var":
        e = rng.uniform(0.01, 0.2, 800).astype(np.float32)
        m = (lc.sinusoid(t, 4.0) + rng.normal(0, 1, 800) * e).astype(np.float32)
    else:
        m = lc.noisy(rng, lc.sinusoid(t, 4.0), 0.03)
        e = np.full(800, 0.05, np.float32) if errs == "const" else None
    P = lc.trial_periods(4.0, n=500)
    r = gpu.FPW(n_bins=15).calc([t], [m], P, np.zeros(1, np.float32),
                                errs=None if e is None else [e])
    assert abs(r[0].params[0] - 4.0) / 4.0 < 0.05


@pytest.mark.parametrize("semantics", ["cuda", "cpu"])
def test_fpw_fast_bins_exact_on_long_baselines(gpu, oracle, semantics):
    """Times near MJD 6e4 with periods of 0.01-0.1 d (up to 6e6 cycles) and a
    period derivative: the chosen form's fast bins, with the reference
    sequence near bin edges, give the plain form's values bit for bit, and
    in CPU semantics the oracle's."""
    rng = np.random.default_rng(17)
    ts, ms, es = [], [], []
    for n in (300, 2000, 4097):
        t = np.sort(rng.uniform(58000.0, 60000.0, n)).astype(np.float32)
        ts.append(t)
        ms.append(lc.noisy(rng, lc.sinusoid(t, 0.0371), 0.05))
        es.append(rng.uniform(0.02, 0.2, n).astype(np.float32))
    P = np.exp(np.linspace(np.log(0.01), np.log(0.1), 900)).astype(np.float32)
    D = np.array([0.0, 1e-7], np.float32)
    for nb in (10, 33):
        a = gpu.FPW(nb, mode="plain", semantics=semantics).periodograms(ts, ms, P, D, errs=es)
        b = gpu.FPW(nb, mode="chosen", semantics=semantics).periodograms(ts, ms, P, D, errs=es)
        np.testing.assert_array_equal(a, b)
        if semantics == "cpu":
            np.testing.assert_array_equal(b, oracle.fpw(ts, ms, P, D, nb, errs=es))


def test_fpw_bls_pipelined_peaks_equal_one_call(gpu):
    """A large 'peaks' request of FPW or BLS runs as PF_ASYNC chunks (packing
    the next chunk and building the last one's results while the GPU runs);
    the result equals one synchronous native call's peak for peak, with and
    without uncertainties.  PF_ASYNC is refused on the periodogram calls
    and after two uncollected calls."""
    from periodfind_b200 import _native as nat
    from periodfind_b200.gpu import unravel_peaks

    rng = np.random.default_rng(12)
    ts = [lc.uniform_times(rng, int(rng.integers(3000, 4097)), 1500.0) for _ in range(80)]
    ms = [lc.noisy(rng, 15.0 + lc.box_eclipse(t, float(rng.uniform(0.5, 10)), depth=0.3,
                                               duty=0.05), 0.05) for t in ts]
    es = [rng.uniform(0.02, 0.3, len(t)).astype(np.float32) for t in ts]
    P = np.exp(np.linspace(np.log(0.2), np.log(60.0), 45000)).astype(np.float32)
    D = np.array([0.0, 1e-6], np.float32)
    assert gpu.FPW._pipelined(ts, P, D)
    for obj in (gpu.FPW(10), gpu.BoxLeastSquares(30, 0.02, 0.3)):
        for e in (es, None):
            got = obj.calc(ts, ms, P, D, errs=e, output="peaks", n_peaks=8, min_distance=3)
            idx, val = obj.peaks(ts, ms, P, D, 8, 3, errs=e)
            want = unravel_peaks(idx, val, P, D, 8)
            assert len(got) == len(want) == len(ts)
            for g, w in zip(got, want):
                assert [(s.params, s.value) for s in g] == [(s.params, s.value) for s in w]
    ctx = nat.default_context(0)
    obj = gpu.FPW(10)
    out = np.empty((2, 50, 1), np.float32)
    P2, Z = np.linspace(1.0, 5.0, 50).astype(np.float32), np.zeros(1, np.float32)
    with ctx.lock:
        assert obj._call(ctx, ctx.lib.pf_fpw, ts[:2], ms[:2], None, P2, Z,
                         obj._flags | nat.PF_ASYNC, nat.ptr(out)) == nat.PF_EINVAL
        idx = np.full((2, 4), -1, np.int64)
        val = np.zeros((2, 4), np.float32)
        for _ in range(2):
            assert obj._call(ctx, ctx.lib.pf_fpw_peaks, ts[:2], ms[:2], None, P2, Z, 4, 1,
                             obj._flags | nat.PF_ASYNC, nat.ptr(idx), nat.ptr(val)) == nat.PF_OK
        assert obj._call(ctx, ctx.lib.pf_fpw_peaks, ts[:2], ms[:2], None, P2, Z, 4, 1,
                         obj._flags | nat.PF_ASYNC, nat.ptr(idx), nat.ptr(val)) == nat.PF_EINVAL
        for _ in range(2):
            ctx.check(ctx.lib.pf_wait(ctx.handle))
    want_idx, want_val = obj.peaks(ts[:2], ms[:2], P2, Z, 4, 1)
    np.testing.assert_array_equal(idx, want_idx)
    np.testing.assert_array_equal(val, want_val)
