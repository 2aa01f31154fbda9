"""The reference's GPU integration expectations (tests/test_periodfind.py:
452-850, 957-1305; tests/test_cpu_standalone.py:992-1155 for 'peaks'),
exercised on the drop-in classes."""

import warnings

import numpy as np
import pytest

from periodfind_b200 import Periodogram, Statistics
import lightcurves as lc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from periodfind_b200 import gpu as g

    return g


ZERO = np.array([0.0], np.float32)


def _detect(obj, true_p, **kw):
    t, m = lc.sine_curve(true_p, n=800, noise=0.02, t_span=200.0)
    res = obj.calc([t], [m], lc.trial_periods(true_p, n=500), ZERO, output="stats", **kw)
    return res[0].params[0]


@pytest.mark.parametrize("mode", ["chosen", "plain"])
def test_known_period_all_algorithms(gpu, mode):
    for obj in (gpu.ConditionalEntropy(15, 10, mode=mode), gpu.AOV(15, mode=mode),
                gpu.LombScargle(mode=mode)):
        got = _detect(obj, 5.0)
        assert abs(got - 5.0) / 5.0 < 0.05, (type(obj).__name__, got)


def test_stats_output_types(gpu):
    t, m = lc.sine_curve(2.5)
    res = gpu.ConditionalEntropy().calc([t], [m], lc.trial_periods(2.5), ZERO)
    assert isinstance(res, list) and len(res) == 1 and isinstance(res[0], Statistics)
    assert res[0].significance > 0
    multi = gpu.ConditionalEntropy().calc([t], [m], np.linspace(1, 10, 200, dtype=np.float32),
                                          ZERO, n_stats=5)
    assert isinstance(multi[0], list) and len(multi[0]) == 5


def test_periodogram_shapes_and_use_max(gpu):
    t, m = lc.sine_curve(3.0)
    P = np.linspace(1, 10, 100, dtype=np.float32)
    D2 = np.array([0.0, 0.001], np.float32)
    pg = gpu.ConditionalEntropy().calc([t], [m], P, D2, output="periodogram")[0]
    assert isinstance(pg, Periodogram) and pg.data.shape == (100, 2) and pg.use_max is False
    assert gpu.AOV().calc([t], [m], P, ZERO, output="periodogram")[0].use_max is True
    assert gpu.LombScargle().calc([t], [m], P, ZERO, output="periodogram")[0].use_max is True
    D5 = np.linspace(-0.01, 0.01, 5, dtype=np.float32)
    assert gpu.ConditionalEntropy().calc([t], [m], P[:50], D5,
                                         output="periodogram")[0].data.shape == (50, 5)


def test_short_lightcurve_all_algorithms(gpu):
    t = np.array([0, 1, 2, 3, 4], np.float32)
    m = np.array([1.0, 0.5, 1.0, 0.5, 1.0], np.float32)
    P = np.linspace(1, 5, 20, dtype=np.float32)
    for cls in (gpu.ConditionalEntropy, gpu.AOV, gpu.LombScargle):
        assert isinstance(cls().calc([t], [m], P, ZERO)[0], Statistics)


def test_center_normalize_warning(gpu):
    t, m = lc.sine_curve(3.0)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        gpu.ConditionalEntropy().calc([t], [m], np.linspace(1, 10, 50, dtype=np.float32), ZERO,
                                      normalize=True, center=True)
    assert any(issubclass(x.category, RuntimeWarning) for x in w)


def test_significance_types(gpu):
    t, m = lc.sine_curve(3.0, n=300)
    for st in ("stdmean", "madmedian"):
        r = gpu.AOV().calc([t], [m], np.linspace(1, 10, 100, dtype=np.float32), ZERO,
                           significance_type=st)
        assert r[0].significance_type == st and r[0].significance > 0


def test_aov_overlap_smoother(gpu):
    t, m = lc.sine_curve(3.0, n=800, noise=0.03, t_span=200.0)
    P = lc.trial_periods(3.0, n=300)
    a = gpu.AOV(10, 1).calc([t], [m], P, ZERO, output="periodogram")[0].data.ravel()
    b = gpu.AOV(10, 3).calc([t], [m], P, ZERO, output="periodogram")[0].data.ravel()
    assert not np.allclose(a, b, atol=1e-6)
    assert np.std(np.diff(b)) < np.std(np.diff(a))
    assert abs(_detect(gpu.AOV(15, 3), 4.0) - 4.0) / 4.0 < 0.05


def test_batched_and_large_grid(gpu):
    curves = [lc.sine_curve(p, seed=i) for i, p in enumerate([2.0, 4.0, 6.0])]
    ts = [c[0] for c in curves]
    ms = [c[1] for c in curves]
    P = np.linspace(1, 10, 5000, dtype=np.float32)
    res = gpu.LombScargle().calc(ts, ms, P, ZERO)
    assert len(res) == 3
    for true_p, r in zip([2.0, 4.0, 6.0], res):
        got = r.params[0]
        assert any(abs(got - c) / c < 0.05 for c in (true_p, true_p / 2, 2 * true_p))


def test_stats_best_matches_periodogram_best(gpu):
    t, m = lc.sine_curve(3.0, n=500, noise=0.02)
    P = lc.trial_periods(3.0, n=300)
    s = gpu.AOV(10).calc([t], [m], P, ZERO, output="stats")[0]
    pg = gpu.AOV(10).calc([t], [m], P, ZERO, output="periodogram")[0]
    assert s.params[0] == pytest.approx(pg.best_params(n=1).params[0])


def test_peaks_output_contract(gpu):
    t, m = lc.sine_curve(5.0, n=800, noise=0.02, t_span=200.0)
    P = lc.trial_periods(5.0, n=500)
    for obj, use_max in ((gpu.ConditionalEntropy(15, 10), False), (gpu.AOV(15), True),
                         (gpu.LombScargle(), True)):
        stats = obj.calc([t], [m], P, ZERO, output="stats")
        peaks = obj.calc([t], [m], P, ZERO, output="peaks", n_peaks=32, min_distance=1)
        assert isinstance(peaks, list) and isinstance(peaks[0], list)
        assert 0 < len(peaks[0]) <= 32 and isinstance(peaks[0][0], Statistics)
        assert stats[0].params[0] == pytest.approx(peaks[0][0].params[0])
        vals = [p.value for p in peaks[0]]
        assert all((a >= b) if use_max else (a <= b) for a, b in zip(vals, vals[1:]))
    D2 = np.array([0.0, 0.001], np.float32)
    pk = gpu.AOV().calc([t], [m], P[:100], D2, output="peaks", n_peaks=16)
    assert len(pk[0][0].params) == 2
    close = gpu.AOV().calc([t], [m], P, ZERO, output="peaks", min_distance=1)
    far = gpu.AOV().calc([t], [m], P, ZERO, output="peaks", min_distance=20)
    assert len(far[0]) <= len(close[0])


def test_lsst_like_cadence(gpu):
    rng = np.random.default_rng(3)
    t = lc.seasonal_times(rng, 600, 3000.0)
    for shape, true_p in (("sine", 0.73), ("eclipse", 2.31)):
        y = lc.sinusoid(t, true_p) if shape == "sine" else lc.v_eclipse(t, true_p)
        m = lc.noisy(rng, y, 0.03)
        P = lc.trial_periods(true_p, n=4000, margin=0.3)
        for obj in (gpu.ConditionalEntropy(), gpu.AOV(15), gpu.LombScargle()):
            if shape == "eclipse" and isinstance(obj, gpu.LombScargle):
                continue
            got = obj.calc([t], [m], P, ZERO)[0].params[0]
            assert any(abs(got - c) / c < 0.01 for c in (true_p, true_p / 2, 2 * true_p)), got


@pytest.mark.parametrize("algo", ["ce", "aov", "ls"])
def test_batch_plan_replays_the_pipeline(algo):
    """A plan (the device pipeline captured as a CUDA graph) gives the direct
    call's periodogram and peaks on two launches in a row, and follows new
    data written into its input buffers in place."""
    import torch

    from periodfind_b200 import _native as nat
    from periodfind_b200.plan import BatchPlan

    rng = np.random.default_rng(5)
    lengths = [30, 300, 1200, 80, 5000, 7]
    ts = [lc.uniform_times(rng, n, 500.0) for n in lengths]
    ms = [lc.normalize(lc.noisy(rng, lc.sinusoid(t, 3.3), 0.1)).astype(np.float32) for t in ts]
    off = np.zeros(len(ts) + 1, np.int64)
    np.cumsum(lengths, out=off[1:])
    d_t = torch.from_numpy(np.concatenate(ts)).cuda()
    d_m = torch.from_numpy(np.concatenate(ms)).cuda()
    P = torch.from_numpy(np.linspace(0.5, 12.0, 700).astype(np.float32)).cuda()
    D = torch.tensor([0.0, 1e-5], dtype=torch.float32, device="cuda")
    shape = (len(ts), 700, 2)
    out = torch.empty(shape, device="cuda")
    pidx = torch.empty((len(ts), 8), dtype=torch.int64, device="cuda")
    pval = torch.empty((len(ts), 8), device="cuda")
    plan = BatchPlan(algo, d_t, d_m, off, P, D, out, n_phase=12, n_mag=8, n_peaks=8,
                     peak_idx=pidx, peak_val=pval)
    ctx = nat.default_context(0)

    def direct():
        ref = torch.empty(shape, device="cuda")
        ri = torch.empty((len(ts), 8), dtype=torch.int64, device="cuda")
        rv = torch.empty((len(ts), 8), device="cuda")
        c = (ctx.handle, d_t.data_ptr(), d_m.data_ptr(), off.ctypes.data, len(ts), P.data_ptr(),
             700, D.data_ptr(), 2)
        with ctx.lock:
            if algo == "ce":
                ctx.check(ctx.lib.pf_ce_dev(*c, 12, 8, 1, 1, nat.PF_MODE_CHOSEN, ref.data_ptr(), 0))
            elif algo == "aov":
                ctx.check(ctx.lib.pf_aov_dev(*c, 12, 1, nat.PF_MODE_CHOSEN, ref.data_ptr(), 0))
            else:
                ctx.check(ctx.lib.pf_ls_dev(*c, nat.PF_MODE_CHOSEN, ref.data_ptr(), 0))
            ctx.check(ctx.lib.pf_find_peaks_dev(ctx.handle, ref.data_ptr(), len(ts), 1400, 8, 1,
                                                0 if algo == "ce" else 1, ri.data_ptr(),
                                                rv.data_ptr(), 0))
        torch.cuda.synchronize()
        return ref, ri, rv

    for _ in range(2):
        out.fill_(-7.0)
        plan.launch()
        torch.cuda.synchronize()
        ref, ri, rv = direct()
        assert torch.equal(out, ref) and torch.equal(pidx, ri) and torch.equal(pval, rv)
    # refill the magnitudes in place: the next launch follows them
    d_m.copy_(torch.from_numpy(np.concatenate(
        [lc.normalize(rng.normal(size=n).astype(np.float32)) for n in lengths])).cuda())
    plan.launch()
    torch.cuda.synchronize()
    ref, ri, rv = direct()
    assert torch.equal(out, ref) and torch.equal(pidx, ri)
    plan.close()


def test_batch_plan_rejects_bad_arguments():
    import ctypes

    from periodfind_b200 import _native as nat

    lib = nat.load()
    h = ctypes.c_void_p()
    off = np.array([0, 3], np.int64)
    rc = lib.pf_plan_create(0, 7, None, None, off.ctypes.data, 1, None, 1, None, 1, 10, 10, 1, 1,
                            nat.PF_MODE_CHOSEN, None, 0, 1, None, None, ctypes.byref(h))
    assert rc == nat.PF_EINVAL and b"algo" in lib.pf_plan_error(None)


def _stats_equal(a, b, data=None, grid=None):
    """Same statistics; the same best cells, except that among cells of equal
    value (a tie) numpy's pick is its partition order and the device takes
    the lowest index -- then the device's cell must hold that value too."""
    for x, y in zip(a if isinstance(a, list) else [a], b if isinstance(b, list) else [b]):
        for f in ("value", "mean", "std", "median", "mad"):
            gx, gy = getattr(x, f), getattr(y, f)
            assert type(gx) is type(gy) and (gx == gy or (np.isnan(gx) and np.isnan(gy))), \
                (f, gx, gy)
        assert [type(p) for p in x.params] == [type(p) for p in y.params]
        if x.params != y.params:
            P, D = grid
            i = int(np.nonzero(P == x.params[0])[0][0])
            j = int(np.nonzero(D == x.params[1])[0][0])
            assert data[i, j] == x.value, "device pick is not a tie of the best value"


@pytest.mark.parametrize("algo", ["ce", "aov", "ls"])
@pytest.mark.parametrize("n_stats", [1, 5])
def test_stats_on_device_equal_numpy(gpu, algo, n_stats):
    """calc(output='stats') computes the statistics on the device; they equal
    the reference's numpy statistics_from_data on the same periodogram bit
    for bit (float32 mean / std in numpy's summation order, exact median /
    MAD, the same best cells and types)."""
    rng = np.random.default_rng(31)
    ts, ms = [], []
    for n in (300, 47, 1200, 9):
        t = lc.uniform_times(rng, n, 300.0)
        ts.append(t)
        ms.append(lc.noisy(rng, lc.sinusoid(t, float(rng.uniform(1, 9)), amp=0.3, offset=15.0),
                           0.05))
    make = {"ce": lambda: gpu.ConditionalEntropy(), "aov": lambda: gpu.AOV(12),
            "ls": lambda: gpu.LombScargle()}[algo]
    obj = make()
    # Rows of up to 8192 cells are sorted in shared memory; longer rows
    # (9000 here) take the radix-selection path.
    for n_per, pdts in ((1001, [0.0]), (1000, [0.0]), (400, [0.0, 1e-5]), (9000, [0.0])):
        if obj._use_max and len(pdts) > 1:
            continue  # the reference's largest-n pick is numpy's partition order there
        P = np.linspace(0.7, 11.0, n_per).astype(np.float32)
        D = np.array(pdts, np.float32)
        got = obj.calc(ts, ms, P, D, output="stats", n_stats=n_stats)
        pgs = obj.calc(ts, ms, P, D, output="periodogram")
        with warnings.catch_warnings():
            # numpy's std of an AOV row holding inf (a curve shorter than
            # its bins) warns; the device statistics carry the same NaN.
            warnings.simplefilter("ignore", RuntimeWarning)
            want = [Statistics.statistics_from_data(pg.data, [P, D], obj._use_max, n=n_stats)
                    for pg in pgs]
        for g, w, pg in zip(got, want, pgs):
            _stats_equal(g, w, pg.data, (P, D))


def test_stats_on_device_nan_rows_and_host_cases(gpu):
    """An empty curve (CE NaN row) gives NaN statistics as numpy does; the
    largest-n pick with several period derivatives keeps the numpy path."""
    t, m = lc.sine_curve(2.0)
    m = lc.normalize(m).astype(np.float32)
    P = np.linspace(1.0, 5.0, 300).astype(np.float32)
    # normalize=False: an empty curve reaches the kernels (normalising it
    # raises, as in the reference) and its CE row is NaN.
    kw = dict(normalize=False)
    got = gpu.ConditionalEntropy().calc([t, np.zeros(0, np.float32)],
                                        [m, np.zeros(0, np.float32)], P,
                                        np.zeros(1, np.float32), output="stats", **kw)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        pgs = gpu.ConditionalEntropy().calc([t, np.zeros(0, np.float32)],
                                            [m, np.zeros(0, np.float32)], P,
                                            np.zeros(1, np.float32), output="periodogram", **kw)
        want = [Statistics.statistics_from_data(pg.data, [P, np.zeros(1, np.float32)], False)
                for pg in pgs]
    _stats_equal(got[0], want[0], pgs[0].data, (P, np.zeros(1, np.float32)))
    assert np.isnan(got[1].mean) and np.isnan(got[1].median) and np.isnan(got[1].mad)
    assert np.isnan(want[1].mean) and np.isnan(want[1].median)
    D2 = np.array([0.0, 1e-5], np.float32)
    a = gpu.AOV().calc([t], [m], P, D2, output="stats")
    pg = gpu.AOV().calc([t], [m], P, D2, output="periodogram")[0]
    _stats_equal(a[0], Statistics.statistics_from_data(pg.data, [P, D2], True))


def test_peaks_output_chunked_equals_one_call(gpu):
    """Large 'peaks' requests run in chunks overlapped with result building;
    the result equals a single native call's peak for peak."""
    from periodfind_b200.gpu import unravel_peaks

    rng = np.random.default_rng(8)
    ts = [lc.uniform_times(rng, 4096, 2000.0) for _ in range(256)]
    ms = [lc.noisy(rng, lc.sinusoid(t, float(rng.uniform(0.5, 10))), 0.05) for t in ts]
    P = np.exp(np.linspace(np.log(0.1), np.log(100.0), 20000)).astype(np.float32)
    D = np.zeros(1, np.float32)
    obj = gpu.AOV(15)
    got = obj.calc(ts, ms, P, D, output="peaks", n_peaks=8)
    idx, val = obj.peaks(ts, ms, P, D, 8)
    want = unravel_peaks(idx, val, P, D, 8)
    assert len(got) == len(want) == 256
    for g, w in zip(got, want):
        assert [(s.params, s.value) for s in g] == [(s.params, s.value) for s in w]


def test_async_peak_calls_equal_synchronous_calls(gpu):
    """PF_ASYNC peak calls queue their work and return; pf_wait collects
    them oldest first into the arrays each call was given.  Two may be
    pending at once; the results equal the synchronous calls' bit for bit
    (CE, AOV, LS)."""
    from periodfind_b200 import _native as nat

    rng = np.random.default_rng(21)
    P = np.exp(np.linspace(np.log(0.2), np.log(50.0), 3000)).astype(np.float32)
    D = np.array([0.0, 1e-6], np.float32)
    batches = []
    for k in range(3):
        ts = [lc.uniform_times(rng, int(rng.integers(20, 900)), 500.0) for _ in range(40 + k)]
        ms = [lc.noisy(rng, lc.sinusoid(t, float(rng.uniform(0.5, 10))), 0.05) for t in ts]
        batches.append((ts, ms))
    ctx = nat.default_context(0)
    for obj in (gpu.ConditionalEntropy(10, 10), gpu.AOV(12), gpu.LombScargle()):
        prep = [(ts, [lc.normalize(m) for m in ms] if isinstance(obj, gpu.ConditionalEntropy)
                 else ms) for ts, ms in batches]
        want = [obj.peaks(ts, ms, P, D, 16, 2) for ts, ms in prep]
        got = []
        with ctx.lock:
            for k, (ts, ms) in enumerate(prep):
                b = nat.CurveBatch(ts, ms)
                idx = np.full((b.n, 16), -7, np.int64)
                val = np.full((b.n, 16), 7.0, np.float32)
                ctx.check(obj._native_peaks(ctx, b, P, D, 16, 2, idx, val, nat.PF_ASYNC))
                got.append((idx, val))
                if k == 1:  # two pending: collect the first
                    ctx.check(ctx.lib.pf_wait(ctx.handle))
            ctx.check(ctx.lib.pf_wait(ctx.handle))
            ctx.check(ctx.lib.pf_wait(ctx.handle))
        for (gi, gv), (wi, wv) in zip(got, want):
            np.testing.assert_array_equal(gi, wi)
            np.testing.assert_array_equal(gv, wv)


def test_async_call_rules(gpu):
    """pf_wait with nothing pending, a third pending call, PF_ASYNC outside
    the peak calls and PF_ASYNC with PF_TIMING are refused with PF_EINVAL;
    an empty batch is a pending call with nothing to copy."""
    from periodfind_b200 import _native as nat

    ctx = nat.Context(0)
    try:
        lib, h = ctx.lib, ctx.handle
        assert lib.pf_wait(h) == nat.PF_EINVAL
        rng = np.random.default_rng(2)
        ts = [lc.uniform_times(rng, 300, 100.0) for _ in range(8)]
        ms = [lc.noisy(rng, lc.sinusoid(t, 3.0), 0.05) for t in ts]
        b = nat.CurveBatch(ts, ms)
        P = np.linspace(0.5, 10, 500).astype(np.float32)
        D = np.zeros(1, np.float32)
        idx = [np.full((8, 4), -1, np.int64) for _ in range(3)]
        val = [np.zeros((8, 4), np.float32) for _ in range(3)]
        flags = nat.PF_MODE_CHOSEN | nat.PF_ASYNC

        def call(k, fl=flags):
            return lib.pf_ls_peaks(h, *b.args(), nat.ptr(P), len(P), nat.ptr(D), len(D), 4, 1,
                                   fl, nat.ptr(idx[k]), nat.ptr(val[k]))

        assert call(0) == nat.PF_OK and call(1) == nat.PF_OK
        assert call(2) == nat.PF_EINVAL
        assert lib.pf_wait(h) == nat.PF_OK and lib.pf_wait(h) == nat.PF_OK
        assert lib.pf_wait(h) == nat.PF_EINVAL
        np.testing.assert_array_equal(idx[0], idx[1])
        assert (idx[0][:, 0] >= 0).all()
        assert call(0, flags | nat.PF_TIMING) == nat.PF_EINVAL
        out = np.zeros((8, len(P), 1), np.float32)
        assert lib.pf_ls(h, *b.args(), nat.ptr(P), len(P), nat.ptr(D), len(D), flags,
                         nat.ptr(out)) == nat.PF_EINVAL
        empty = nat.CurveBatch([], [])
        assert lib.pf_ls_peaks(h, *empty.args(), nat.ptr(P), len(P), nat.ptr(D), len(D), 4, 1,
                               flags, nat.ptr(idx[2]), nat.ptr(val[2])) == nat.PF_OK
        assert lib.pf_wait(h) == nat.PF_OK
        assert lib.pf_wait(h) == nat.PF_EINVAL
    finally:
        ctx.close()


def test_chunked_peaks_prepare_magnitudes_per_chunk(gpu):
    """A pipelined 'peaks' batch prepares the magnitudes chunk by chunk; CE's
    normalisation per chunk equals the whole batch's, and the centre /
    normalise conflict (periodfind/_utils.py:29-37) warns once per call."""
    from periodfind_b200._utils import prepare_magnitudes
    from periodfind_b200.gpu import unravel_peaks

    rng = np.random.default_rng(12)
    ts = [lc.uniform_times(rng, 4096, 2000.0) for _ in range(128)]
    ms = [lc.noisy(rng, 15.0 + 0.3 * lc.sinusoid(t, float(rng.uniform(0.5, 10))), 0.05)
          for t in ts]
    P = np.exp(np.linspace(np.log(0.1), np.log(100.0), 40000)).astype(np.float32)
    D = np.zeros(1, np.float32)
    obj = gpu.ConditionalEntropy(10, 10)
    got = obj.calc(ts, ms, P, D, output="peaks", n_peaks=8)
    idx, val = obj.peaks(ts, prepare_magnitudes(ms, False, True), P, D, 8)
    want = unravel_peaks(idx, val, P, D, 8)
    assert len(got) == 128
    for g, w in zip(got, want):
        assert [(s.params, s.value) for s in g] == [(s.params, s.value) for s in w]
    with warnings.catch_warnings(record=True) as rec:
        warnings.simplefilter("always")
        got = obj.calc(ts, ms, P, D, output="peaks", n_peaks=8, center=True, normalize=True)
    assert sum(issubclass(r.category, RuntimeWarning) for r in rec) == 1
    idx, val = obj.peaks(ts, [m - np.mean(m) for m in ms], P, D, 8)
    want = unravel_peaks(idx, val, P, D, 8)
    for g, w in zip(got, want):
        assert [(s.params, s.value) for s in g] == [(s.params, s.value) for s in w]


def test_ce_magnitudes_outside_unit_interval_run_memory_safely(gpu):
    """CE magnitudes are bin coordinates meant to lie in [0, 1), but the
    reference's own tests run CE on centred magnitudes
    (tests/test_periodfind.py:535-546), so values outside are accepted.
    Raw (15 +- 0.3), centred, NaN and >= 1 magnitudes give a periodogram of
    the right shape; a centred curve's negative values fall in magnitude bin
    0, which the CPU-semantics oracle (Rust's saturating cast) reproduces."""
    from oracle import oracle as O

    t, m = lc.sine_curve(2.0, n=300)
    P = np.linspace(1.0, 5.0, 200).astype(np.float32)
    Z = np.zeros(1, np.float32)
    ce = gpu.ConditionalEntropy()
    raw = (15.0 + 0.3 * m).astype(np.float32)
    odd = lc.normalize(m).astype(np.float32)
    odd[7], odd[9] = np.nan, 1.0
    for mags in (raw, odd, (m - np.mean(m)).astype(np.float32)):
        for output in ("stats", "periodogram", "peaks"):
            assert len(ce.calc([t], [mags], P, Z, output=output, normalize=False)) == 1
    cen = (0.3 * (m - np.mean(m))).astype(np.float32)
    got = gpu.ConditionalEntropy(semantics="cpu").periodograms([t], [cen], P, Z)
    np.testing.assert_allclose(got, O.ce([t], [cen], P, Z), rtol=2e-6)


def test_preparation_fused_into_packing_is_bit_exact():
    """PF_HOST_NORMALIZE / PF_HOST_CENTER prepare the magnitudes while the
    library packs them: the periodograms equal those of magnitudes prepared
    by numpy first, bit for bit (CE normalised, LS centred, AOV centred),
    with a constant and a one-point curve among them, and enough points
    (~90 000) that the packing runs on several of the context's threads."""
    from periodfind_b200 import _native as nat
    from periodfind_b200 import gpu

    rng = np.random.default_rng(61)
    ts, ms = [], []
    for n in (1, 7, 8, 9, 129, 300, 1025, 4097) + (2000,) * 40:
        t = lc.uniform_times(rng, n, 200.0)
        ts.append(t)
        ms.append(lc.noisy(rng, lc.sinusoid(t, float(rng.uniform(1, 4)), 0.3, 0.0, 15.0), 0.05))
    ms[3][:] = 7.5
    P = np.linspace(0.5, 6.0, 257).astype(np.float32)
    D = np.array([0.0, 1e-5], np.float32)
    for obj, center in ((gpu.ConditionalEntropy(10, 10), False), (gpu.LombScargle(), True),
                        (gpu.AOV(15), True)):
        with np.errstate(all="ignore"):
            want = obj.periodograms(ts, [np.asarray(m) for m in
                                         (lc.center(x) if center else lc.normalize(x)
                                          for x in ms)], P, D)
            got = obj.periodograms(ts, ms, P, D, _extra=nat.PF_HOST_CENTER if center
                                   else nat.PF_HOST_NORMALIZE)
        np.testing.assert_array_equal(got, want)
