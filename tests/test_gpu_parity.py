"""GPU parity tests: the CUDA path (through the C ABI) against the oracle
(the reference's CPU arithmetic), against the reference's own CUDA build
(when oracle/_ref is present), and between the plain and chosen forms.

Tolerances, written per comparison:
  * CPU semantics vs the oracle
      AOV plain: bit-exact (same bins, same f32 adds in the same order).
      CE: rtol 2e-6 (bins are identical; logf on the GPU and in glibc may
          differ by an ulp).
      LS: |diff| <= 2e-5 * max|P| + 2e-5 * |P| (sinf/cosf ulp differences
          accumulated over the curve).
  * chosen vs plain (same semantics): CE and LS bit-exact (the exact fold
    is the reference fold's quotient without a divide); AOV chosen uses the
    exact fixed-point accumulator and must match the FP64 statistic on the
    same bins to rtol 1e-6.
  * CUDA semantics vs the reference CUDA build: CE rtol 1e-5 (the reference
    sums rows in atomic order), AOV rtol 2e-4 and LS rtol 1e-4 with an
    absolute floor (the reference's f32 sums are order-dependent).
"""

import numpy as np
import pytest

import lightcurves as lc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def gpu():
    from periodfind_b200 import gpu as g

    return g


def _grid(n_per=300, pdts=(0.0,), lo=0.5, hi=10.0):
    return (np.linspace(lo, hi, n_per, dtype=np.float32), np.array(pdts, np.float32))


def _ragged(seed=7, lengths=(1, 2, 5, 31, 32, 33, 255, 256, 257, 1023, 1024, 1025, 2049)):
    rng = np.random.default_rng(seed)
    ts, ms = [], []
    for n in lengths:
        t = lc.uniform_times(rng, n, 400.0)
        p = float(rng.uniform(0.5, 10))
        ms.append(lc.noisy(rng, lc.sinusoid(t, p, amp=0.3, offset=15.0), 0.05))
        ts.append(t)
    return ts, ms


def _ls_close(a, b, rel=2e-5):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = np.nanmax(np.abs(b)) if b.size else 1.0
    assert np.all(np.abs(a - b) <= rel * scale + rel * np.abs(b)), np.nanmax(np.abs(a - b))


# ------------------------------------------------- CPU semantics vs oracle


@pytest.mark.parametrize("mode", ["plain", "chosen"])
def test_ce_cpu_semantics_vs_oracle(gpu, oracle, mode):
    ts, ms = _ragged()
    ms = [lc.normalize(m) if len(m) > 1 else np.full(1, 0.5, np.float32) for m in ms]
    P, D = _grid(pdts=(0.0, 1e-4, -3e-4))
    got = gpu.ConditionalEntropy(10, 10, mode=mode, semantics="cpu").periodograms(ts, ms, P, D)
    want = oracle.ce(ts, ms, P, D, 10, 10)
    np.testing.assert_allclose(got, want, rtol=2e-6, atol=0)


def test_aov_plain_cpu_semantics_bit_exact(gpu, oracle):
    ts, ms = _ragged()
    P, D = _grid(pdts=(0.0, 1e-4))
    got = gpu.AOV(15, mode="plain", semantics="cpu").periodograms(ts, ms, P, D)
    want = oracle.aov(ts, ms, P, D, 15)
    np.testing.assert_array_equal(got, want)


def test_aov_chosen_matches_fp64_statistic(gpu, oracle):
    ts, ms = _ragged()
    keep = [i for i, t in enumerate(ts) if len(t) >= 16]
    ts = [ts[i] for i in keep]
    ms = [ms[i] for i in keep]
    P, D = _grid(pdts=(0.0, 1e-4))
    got = gpu.AOV(15, mode="chosen", semantics="cpu").periodograms(ts, ms, P, D)
    want = oracle.aov_f64(ts, ms, P, D, 15)
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-6 * np.max(np.abs(want)))


@pytest.mark.parametrize("mode", ["plain", "chosen"])
def test_ls_cpu_semantics_vs_oracle(gpu, oracle, mode):
    ts, ms = _ragged()
    ms = [lc.center(m) for m in ms]
    P, D = _grid(pdts=(0.0, 1e-4))
    got = gpu.LombScargle(mode=mode, semantics="cpu").periodograms(ts, ms, P, D)
    want = oracle.ls(ts, ms, P, D)
    _ls_close(got, want)


@pytest.mark.parametrize("po,mo", [(3, 1), (1, 2), (2, 3)])
def test_ce_overlap_vs_oracle(gpu, oracle, po, mo):
    t, m = lc.sine_curve(3.0, n=600)
    m = lc.normalize(m)
    P, D = _grid(200)
    got = gpu.ConditionalEntropy(10, 10, po, mo, semantics="cpu").periodograms([t], [m], P, D)
    want = oracle.ce([t], [m], P, D, 10, 10, po, mo)
    np.testing.assert_allclose(got, want, rtol=2e-6)


@pytest.mark.parametrize("mode", ["plain", "chosen"])
def test_aov_overlap_vs_oracle(gpu, oracle, mode):
    t, m = lc.sine_curve(4.0, n=600)
    P, D = _grid(200)
    got = gpu.AOV(10, 3, mode=mode, semantics="cpu").periodograms([t], [m], P, D)
    if mode == "plain":
        np.testing.assert_array_equal(got, oracle.aov([t], [m], P, D, 10, 3))
    else:
        want = oracle.aov_f64([t], [m], P, D, 10, 3)
        np.testing.assert_allclose(got, want, rtol=1e-6)


def test_ce_custom_bins_vs_oracle(gpu, oracle):
    t, m = lc.eclipse_curve(2.5, n=600)
    m = lc.normalize(m)
    P, D = _grid(200)
    got = gpu.ConditionalEntropy(15, 10, semantics="cpu").periodograms([t], [m], P, D)
    np.testing.assert_allclose(got, oracle.ce([t], [m], P, D, 15, 10), rtol=2e-6)
    got = gpu.ConditionalEntropy(20, 5, 2, 2, semantics="cpu").periodograms([t], [m], P, D)
    np.testing.assert_allclose(got, oracle.ce([t], [m], P, D, 20, 5, 2, 2), rtol=2e-6)


# ------------------------------------------------------- chosen vs plain


@pytest.mark.parametrize("sem", ["cuda", "cpu"])
def test_chosen_equals_plain_ce_ls(gpu, sem):
    ts, ms = _ragged(seed=3)
    msn = [lc.normalize(m) if len(m) > 1 else np.full(1, 0.5, np.float32) for m in ms]
    P, D = _grid(500, pdts=(0.0, 2e-4))
    a = gpu.ConditionalEntropy(mode="plain", semantics=sem).periodograms(ts, msn, P, D)
    b = gpu.ConditionalEntropy(mode="chosen", semantics=sem,
                               reference_stats=True).periodograms(ts, msn, P, D)
    np.testing.assert_array_equal(a, b)
    msc = [lc.center(m) for m in ms]
    a = gpu.LombScargle(mode="plain", semantics=sem).periodograms(ts, msc, P, D)
    b = gpu.LombScargle(mode="chosen", semantics=sem, fold="exact").periodograms(ts, msc, P, D)
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("pdts", [(0.0,), (0.0, 1e-6, -2e-5)])
def test_bin_kernel_occupancy_exact_at_scale(gpu, pdts):
    """The chosen CE kernel's bins (FP64/integer bin arithmetic with the
    reference's sequence near edges) against the plain kernel's reference
    fold: identical CE values over ~1.2e9 evaluations, i.e. identical
    histograms, including long baselines (MJD-like times, short periods)."""
    import lightcurves as lc2

    ts, ms = lc2.mixed_signal_batch(48, 4096, 1234)
    rng = np.random.default_rng(5)
    for k in range(8):  # long-baseline curves: t ~ 5.9e4 days
        t = np.sort(rng.uniform(58000.0, 60000.0, 4096)).astype(np.float32)
        ts.append(t)
        ms.append(lc2.noisy(rng, lc2.sinusoid(t, 0.123 + 0.01 * k), 0.05))
    msn = [lc2.normalize(m) for m in ms]
    P = np.exp(np.linspace(np.log(0.05), np.log(100.0), 1500)).astype(np.float32)
    D = np.array(pdts, np.float32)
    for sem in ("cuda", "cpu"):
        a = gpu.ConditionalEntropy(mode="plain", semantics=sem).periodograms(ts, msn, P, D)
        b = gpu.ConditionalEntropy(mode="chosen", semantics=sem,
                                   reference_stats=True).periodograms(ts, msn, P, D)
        np.testing.assert_array_equal(a, b)
        # the chosen form's own statistic from the same bins: within 1e-5
        f = gpu.ConditionalEntropy(mode="chosen", semantics=sem).periodograms(ts, msn, P, D)
        np.testing.assert_allclose(f, a, rtol=1e-5)
        a = gpu.ConditionalEntropy(15, 7, mode="plain", semantics=sem).periodograms(ts[:8], msn[:8], P, D)
        b = gpu.ConditionalEntropy(15, 7, mode="chosen", semantics=sem,
                                   reference_stats=True).periodograms(ts[:8], msn[:8], P, D)
        np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("sem", ["cuda", "cpu"])
def test_chosen_statistics_from_same_bins(gpu, sem):
    """The chosen form's divide-free CE / AOV statistics from the same bins:
    CE within 1e-5 of the plain form; AOV within 1e-9 of the chosen form's
    reference-sequence statistic (both FP64 over exact fixed-point sums; the
    plain AOV keeps the reference's f32 sums, which cancel for raw
    magnitudes near 15)."""
    ts, ms = _ragged(seed=8)
    msn = [lc.normalize(m) if len(m) > 1 else np.full(1, 0.5, np.float32) for m in ms]
    P, D = _grid(700, pdts=(0.0, 3e-5))
    for n_phase, n_mag in ((10, 10), (12, 7), (5, 20)):
        a = gpu.ConditionalEntropy(n_phase, n_mag, mode="plain", semantics=sem).periodograms(
            ts, msn, P, D)
        b = gpu.ConditionalEntropy(n_phase, n_mag, mode="chosen", semantics=sem).periodograms(
            ts, msn, P, D)
        np.testing.assert_allclose(b, a, rtol=1e-5)
    keep = [i for i, t in enumerate(ts) if len(t) >= 16]
    tk, mk = [ts[i] for i in keep], [ms[i] for i in keep]
    for n_phase in (15, 10, 3):
        a = gpu.AOV(n_phase, mode="chosen", semantics=sem,
                    reference_stats=True).periodograms(tk, mk, P, D)
        b = gpu.AOV(n_phase, mode="chosen", semantics=sem).periodograms(tk, mk, P, D)
        np.testing.assert_allclose(b, a, rtol=1e-9, atol=1e-9 * np.abs(a).max())


def test_ls_split_precision_phase_is_more_accurate(gpu, oracle):
    """The chosen LS phase (split-precision FP32) against the FP64 oracle:
    at least as close as the reference's f32-rounded fold, point by point
    for >= 99% of the grid, and within 1e-4 of it everywhere."""
    rng = np.random.default_rng(8)
    ts, ms = [], []
    for k in range(4):
        t = lc.seasonal_times(rng, 1500, 3000.0)
        ts.append(t)
        ms.append(lc.center(lc.noisy(rng, 0.3 * np.sin(2 * np.pi * t * rng.uniform(0.1, 15)), 0.05)))
    f = np.linspace(0.01, 20.0, 4000)
    P = (1.0 / f).astype(np.float32)
    for D in (np.zeros(1, np.float32), np.array([0.0, 1e-7], np.float32)):
        truth = oracle.ls_f64(ts, ms, P, D)
        ref = gpu.LombScargle(mode="plain", semantics="cpu").periodograms(ts, ms, P, D)
        df = gpu.LombScargle(mode="chosen", semantics="cpu").periodograms(ts, ms, P, D)
        e_df = np.abs(df - truth)
        e_ref = np.abs(ref - truth)
        scale = np.abs(truth).max()
        assert np.mean(e_df <= e_ref + 1e-6 * scale) >= 0.99
        _ls_close(df, ref, rel=1e-4)


def test_exact_fold_long_baseline(gpu, oracle):
    """Times ~ MJD 6e4 with short periods (1e5..1e6 cycles): the chosen fold
    still reproduces the divide bit for bit (bins identical => CE equal)."""
    rng = np.random.default_rng(11)
    t = np.sort(rng.uniform(58000.0, 60000.0, 2000)).astype(np.float32)
    m = lc.normalize(lc.noisy(rng, lc.sinusoid(t, 0.0371), 0.05))
    P = np.exp(np.linspace(np.log(0.01), np.log(0.1), 700)).astype(np.float32)
    D = np.array([0.0, 1e-7], np.float32)
    a = gpu.ConditionalEntropy(mode="plain", semantics="cpu").periodograms([t], [m], P, D)
    b = gpu.ConditionalEntropy(mode="chosen", semantics="cpu",
                               reference_stats=True).periodograms([t], [m], P, D)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_allclose(b, oracle.ce([t], [m], P, D), rtol=2e-6)
    f = gpu.ConditionalEntropy(mode="chosen", semantics="cpu").periodograms([t], [m], P, D)
    np.testing.assert_allclose(f, a, rtol=1e-5)


# ----------------------------------------------------- peaks on the device


@pytest.mark.parametrize("algo", ["ce", "aov", "ls"])
@pytest.mark.parametrize("n_peaks,min_distance", [(32, 1), (8, 3), (16, 20), (1, 1)])
def test_peaks_match_oracle_on_same_periodogram(gpu, oracle, algo, n_peaks, min_distance):
    ts, ms = _ragged(seed=5, lengths=(40, 300, 700))
    P, D = _grid(2500, pdts=(0.0, 1e-4))  # 5000 cells: crosses the 2048-sample chunk
    if algo == "ce":
        obj, ms, use_max = gpu.ConditionalEntropy(), [lc.normalize(m) for m in ms], False
    elif algo == "aov":
        obj, use_max = gpu.AOV(), True
    else:
        obj, ms, use_max = gpu.LombScargle(), [lc.center(m) for m in ms], True
    pg = obj.periodograms(ts, ms, P, D)
    idx, val = obj.peaks(ts, ms, P, D, n_peaks, min_distance)
    oi, ov = oracle.find_top_peaks_batched(pg, n_peaks, min_distance, use_max)
    np.testing.assert_array_equal(idx, oi)
    np.testing.assert_array_equal(val, ov)


def test_peaks_golden_vectors_on_device(gpu, oracle):
    import json
    import os

    path = os.path.join(os.path.dirname(__file__), "golden", "peaks_golden.json")
    for case in json.load(open(path))["cases"]:
        data = np.array(case["data"], np.float32).reshape(1, -1, 1)
        if data.size == 0:
            data = np.zeros((1, 0, 1), np.float32)
        idx, val = gpu.find_top_peaks_batched(data, case["n_peaks"], case["min_distance"],
                                              case["use_max"])
        oi, ov = oracle.find_top_peaks_batched(data, case["n_peaks"], case["min_distance"],
                                               case["use_max"])
        np.testing.assert_array_equal(idx, oi, err_msg=case["name"])
        np.testing.assert_array_equal(val, ov, err_msg=case["name"])
        if case["expect_idx"] is not None:
            k = len(case["expect_idx"])
            assert idx[0, :k].tolist() == case["expect_idx"], case["name"]


# ------------------------------------------------- reference CUDA build


def _ref_or_skip(oracle):
    if not oracle.ref_available():
        pytest.skip("oracle/_ref/libpfref.so not built (needs the reference checkout)")


def test_ce_vs_reference_cuda(gpu, oracle):
    _ref_or_skip(oracle)
    ts, ms = _ragged(seed=9)
    ms = [lc.normalize(m) if len(m) > 1 else np.full(1, 0.5, np.float32) for m in ms]
    P, D = _grid(400, pdts=(0.0, 1e-4, -1e-3))
    want = oracle.ref_cuda("ce", ts, ms, P, D, n_phase=10, n_mag=10)
    for mode in ("plain", "chosen"):
        got = gpu.ConditionalEntropy(mode=mode).periodograms(ts, ms, P, D)
        np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-7)


def test_aov_vs_reference_cuda(gpu, oracle):
    """AOV against the reference CUDA build on a ragged batch.  The bins are
    the reference's count for count (tests/test_gpu_bins.py compares them
    bin by bin); the values then differ only by the f32 summation order of
    the bin sums, which the reference adds with shared float atomics in no
    fixed order.  Both are held to the FP64 statistic on the same bins: the
    chosen form within 1e-5 relative, the plain form no further from it than
    the same f32 statistic summed in point order as the reference's Rust
    path sums it (the oracle; the plain form adds in that order too), on
    normalised magnitudes and on 15 +- 0.3 raw magnitudes whose f32 sums of
    squares cancel; the reference CUDA build's own error is printed beside
    them.  All at the 99th percentile over cells."""
    _ref_or_skip(oracle)
    ts, ms = _ragged(seed=9, lengths=(64, 300, 1025, 4096, 4097, 6000))
    P, D = _grid(400, pdts=(0.0, 1e-4))
    for mags in ([lc.normalize(m) for m in ms], ms):
        want = oracle.ref_cuda("aov", ts, mags, P, D, n_phase=15)
        truth = oracle.aov_f64(ts, mags, P, D, 15, fused_tcorr=True)
        scale = np.abs(truth).max(axis=(1, 2), keepdims=True)
        rel = lambda x: np.abs(x - truth) / (np.abs(truth) + 1e-6 * scale)
        # Cells whose oracle bins (IEEE divide) differ from the reference's
        # (fast-math divide) have another FP64 truth: the largest errors are
        # compared over the 99% closest cells.
        e_ref = np.quantile(rel(want), 0.99)
        e_seq = np.quantile(rel(oracle.aov(ts, mags, P, D, 15)), 0.99)
        chosen = gpu.AOV(15, mode="chosen").periodograms(ts, mags, P, D)
        plain = gpu.AOV(15, mode="plain").periodograms(ts, mags, P, D)
        e_plain = np.quantile(rel(plain), 0.99)
        print(f"\nAOV 99th-percentile error vs FP64: chosen {np.quantile(rel(chosen), 0.99):.2e}"
              f", plain {e_plain:.2e}, point-order f32 {e_seq:.2e}, reference {e_ref:.2e}")
        assert np.quantile(rel(chosen), 0.99) <= 1e-5
        assert e_plain <= 1.25 * e_seq + 1e-6


def test_ls_vs_reference_cuda(gpu, oracle):
    _ref_or_skip(oracle)
    ts, ms = _ragged(seed=9)
    ms = [lc.center(m) for m in ms]
    P, D = _grid(400, pdts=(0.0, 1e-4))
    want = oracle.ref_cuda("ls", ts, ms, P, D)
    for mode in ("plain", "chosen"):
        got = gpu.LombScargle(mode=mode).periodograms(ts, ms, P, D)
        _ls_close(got, want, rel=1e-4)


# ----------------------------------------------------------- edge cases


def test_empty_and_single_point_curves(gpu, oracle):
    e = np.zeros(0, np.float32)
    one = np.array([3.0], np.float32)
    P, D = _grid(50)
    ce = gpu.ConditionalEntropy(semantics="cpu").periodograms([e, one], [e, one * 0 + 0.5], P, D)
    assert np.all(np.isnan(ce[0]))
    np.testing.assert_allclose(ce[1], oracle.ce([one], [one * 0 + 0.5], P, D)[0], rtol=1e-6)
    aov = gpu.AOV(semantics="cpu").periodograms([e], [e], P, D)
    assert np.all(aov == 0)
    ls = gpu.LombScargle(semantics="cpu").periodograms([e], [e], P, D)
    assert np.all(ls == 0)


def test_nonfinite_times_rejected(gpu):
    from periodfind_b200._native import PeriodfindError

    t = np.array([0.0, np.nan, 2.0], np.float32)
    with pytest.raises(PeriodfindError, match="finite"):
        gpu.AOV().periodograms([t], [t * 0], *_grid(10))


def test_zero_period_rejected(gpu):
    from periodfind_b200._native import PeriodfindError

    t = np.arange(10, dtype=np.float32)
    with pytest.raises(PeriodfindError, match="non-zero"):
        gpu.LombScargle().periodograms([t], [t], np.array([1.0, 0.0], np.float32),
                                       np.zeros(1, np.float32))


def test_repeat_calls_grow_and_shrink(gpu, oracle):
    """Context buffers are reused across calls of different sizes."""
    obj = gpu.AOV(semantics="cpu", mode="plain")
    for n_curves, n in [(2, 50), (5, 3000), (1, 10), (3, 700)]:
        ts, ms = _ragged(seed=n, lengths=[n] * n_curves)
        P, D = _grid(123)
        np.testing.assert_array_equal(obj.periodograms(ts, ms, P, D),
                                      oracle.aov(ts, ms, P, D, 10))


def test_device_pointer_entry_points(gpu):
    torch = pytest.importorskip("torch")
    from periodfind_b200 import _native as nat

    ts, ms = _ragged(seed=21, lengths=(10, 333, 1500))
    P, D = _grid(200, pdts=(0.0, 1e-4))
    host = gpu.LombScargle(mode="chosen").periodograms(ts, [lc.center(m) for m in ms], P, D)
    off = np.zeros(len(ts) + 1, np.int64)
    np.cumsum([len(t) for t in ts], out=off[1:])
    dt = torch.from_numpy(np.concatenate(ts)).cuda()
    dm = torch.from_numpy(np.concatenate([lc.center(m) for m in ms])).cuda()
    dp = torch.from_numpy(P).cuda()
    dd = torch.from_numpy(D).cuda()
    out = torch.empty((len(ts), len(P), len(D)), dtype=torch.float32, device="cuda")
    ctx = nat.default_context(0)
    # The work must be ordered on the caller's stream: the default stream
    # (handle 0) and a side stream, each synchronised on its own.
    side = torch.cuda.Stream()
    for st in (torch.cuda.default_stream(), side):
        out.fill_(-1.0)
        torch.cuda.synchronize()
        with ctx.lock:
            ctx.check(ctx.lib.pf_ls_dev(ctx.handle, dt.data_ptr(), dm.data_ptr(),
                                        off.ctypes.data, len(ts), dp.data_ptr(), len(P),
                                        dd.data_ptr(), len(D), nat.PF_MODE_CHOSEN,
                                        out.data_ptr(), st.cuda_stream))
        done = torch.cuda.Event()
        done.record(st)
        done.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), host)


@pytest.mark.parametrize("algo,mode", [("ce", "chosen"), ("ce", "plain"), ("ls", "chosen")])
def test_per_curve_device_timestamps(gpu, algo, mode):
    """PF_TIMING records a start and end stamp per work item; the results are
    unchanged and every curve gets a positive latency no longer than the
    whole launch."""
    torch = pytest.importorskip("torch")
    import time

    from periodfind_b200 import _native as nat

    ts, ms = _ragged(seed=33, lengths=(20, 700, 64, 2000, 5))
    if algo == "ce":
        ms = [lc.normalize(m) for m in ms]
    P, D = _grid(300, pdts=(0.0, 1e-4))
    off = np.zeros(len(ts) + 1, np.int64)
    np.cumsum([len(t) for t in ts], out=off[1:])
    dt = torch.from_numpy(np.concatenate(ts)).cuda()
    dm = torch.from_numpy(np.concatenate(ms)).cuda()
    dp = torch.from_numpy(P).cuda()
    dd = torch.from_numpy(D).cuda()
    ctx = nat.default_context(0)
    flags = nat.PF_MODE_CHOSEN if mode == "chosen" else nat.PF_MODE_PLAIN
    outs = []
    for extra in (0, nat.PF_TIMING):
        out = torch.empty((len(ts), len(P), len(D)), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        with ctx.lock:
            args = (ctx.handle, dt.data_ptr(), dm.data_ptr(), off.ctypes.data, len(ts),
                    dp.data_ptr(), len(P), dd.data_ptr(), len(D))
            if algo == "ce":
                ctx.check(ctx.lib.pf_ce_dev(*args, 10, 10, 1, 1, flags | extra,
                                            out.data_ptr(), 0))
            else:
                ctx.check(ctx.lib.pf_ls_dev(*args, flags | extra, out.data_ptr(), 0))
            torch.cuda.synchronize()
            wall_ns = (time.perf_counter() - t0) * 1e9
            if extra:
                lat = np.zeros(len(ts))
                ctx.check(ctx.lib.pf_curve_latency(ctx.handle, len(ts), lat.ctypes.data))
                bad = np.zeros(len(ts) + 1)
                assert ctx.lib.pf_curve_latency(ctx.handle, len(ts) + 1,
                                                bad.ctypes.data) == nat.PF_EINVAL
        outs.append(out.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])
    assert np.all(lat > 0) and np.all(lat <= wall_ns), lat


def test_autotuned_launch_shapes_change_no_value(gpu):
    """Curves in every length class: the autotuner picks a launch shape per
    class (block size, persistent or one CTA per item); the values equal the
    untuned launch's bit for bit, and the report lists the tuned classes."""
    from periodfind_b200 import _native as nat

    lengths = [10, 40, 63, 64, 100, 255, 256, 700, 1023, 1024, 3000, 4095, 4096, 6000]
    ts, ms = _ragged(seed=41, lengths=lengths)
    msn = [lc.normalize(m) for m in ms]
    P, D = _grid(900, pdts=(0.0, 2e-5))
    ctx = nat.default_context(0)
    for make, mags in ((lambda **k: gpu.ConditionalEntropy(**k), msn),
                       (lambda **k: gpu.AOV(15, **k), ms),
                       (lambda **k: gpu.LombScargle(**k), [lc.center(m) for m in ms])):
        tuned = make(mode="chosen").periodograms(ts, mags, P, D)
        untuned_obj = make(mode="chosen")
        untuned_obj._flags |= nat.PF_NO_TUNE
        np.testing.assert_array_equal(tuned, untuned_obj.periodograms(ts, mags, P, D))
        # Every class in one launch with one shape: the same values.
        one_obj = make(mode="chosen")
        one_obj._flags |= nat.PF_ONE_LAUNCH
        np.testing.assert_array_equal(tuned, one_obj.periodograms(ts, mags, P, D))
    report = ctx.tuning_report()
    for name in ("[0,64)", "[64,256)", "[256,1024)", "[1024,4096)", "[4096,inf)"):
        assert f"class={name}" in report, report
    assert "ce bin" in report and "aov bin" in report and "ls fold-split" in report


def test_shared_histogram_binning_changes_no_value(gpu):
    """The chosen CE / AOV binning with shared histograms and atomics
    (PF_BINS_SHARED; one histogram per warp and period) gives the
    privatised form's values bit for bit, untuned and tuned, on every
    length class it serves and beside the longer classes it leaves to the
    privatised form; both overlaps of one, with and without a period
    derivative; the tuner lists the strategy it kept per class."""
    from periodfind_b200 import _native as nat

    lengths = [1, 2, 5, 10, 31, 32, 33, 63, 64, 100, 255, 256, 257, 700, 1023, 1024, 3000]
    ts, ms = _ragged(seed=43, lengths=lengths)
    msn = [lc.normalize(m) if len(m) > 1 else np.full(1, 0.5, np.float32) for m in ms]
    P, D = _grid(700, pdts=(0.0, 2e-5))
    for make, mags in ((lambda **k: gpu.ConditionalEntropy(**k), msn),
                       (lambda **k: gpu.AOV(15, **k), ms)):
        want = make(mode="chosen").periodograms(ts, mags, P, D)
        for extra in (nat.PF_BINS_SHARED | nat.PF_NO_TUNE, nat.PF_BINS_SHARED):
            obj = make(mode="chosen")
            obj._flags |= extra
            np.testing.assert_array_equal(obj.periodograms(ts, mags, P, D), want)
    report = nat.default_context(0).tuning_report()
    assert "bins=shared-atomic" in report and "bins=privatised" in report, report


@pytest.mark.parametrize("use_max", [True, False])
def test_peaks_adversarial_rows_match_oracle(gpu, oracle, use_max):
    """The device peak search drops extrema that are not better than the
    threshold at the start of their 2048-sample chunk before its serial
    replay.  Rows that stress that rule match the oracle's streaming search
    (rust/src/peaks.rs:18-238) exactly:

    - a rising trend, so the threshold moves in every chunk;
    - heavily quantised values, so extrema tie the threshold;
    - more peaks requested than one chunk has extrema;
    - a long min_distance;
    - constant, NaN and infinite samples."""
    rng = np.random.default_rng(31)
    n = 30000  # 15 chunks
    x = np.linspace(0.0, 5.0, n)
    rows = [
        x + rng.normal(0, 1, n),                      # rising trend
        -x + rng.normal(0, 1, n),                     # falling trend
        np.round(rng.normal(0, 1, n) * 2) / 2,        # coarse quantisation: ties
        np.round(x * 3 + rng.normal(0, 0.5, n)),      # ties on a trend
        np.sin(np.arange(n) * 0.37) + 1e-3 * rng.normal(0, 1, n),
        np.full(n, 2.0),                              # no extrema
        rng.normal(0, 1, n),
    ]
    rows[6][rng.integers(0, n, 50)] = np.nan
    rows[6][rng.integers(0, n, 20)] = np.inf
    rows[6][rng.integers(0, n, 20)] = -np.inf
    data = np.stack(rows).astype(np.float32).reshape(len(rows), n, 1)
    for n_peaks, min_distance in ((1, 1), (32, 1), (32, 7), (700, 1), (40, 3000)):
        idx, val = gpu.find_top_peaks_batched(data, n_peaks, min_distance, use_max)
        oi, ov = oracle.find_top_peaks_batched(data, n_peaks, min_distance, use_max)
        np.testing.assert_array_equal(idx, oi, err_msg=f"{n_peaks} {min_distance}")
        np.testing.assert_array_equal(val, ov, err_msg=f"{n_peaks} {min_distance}")
