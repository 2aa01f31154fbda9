"""CPU tests of the host-side code: input helpers, result containers, the
GPU classes' argument handling before any device work, and the C ABI
library's exports (no GPU compute)."""

import ctypes
import os
import re
import warnings

import numpy as np
import pytest

from periodfind_b200 import Periodogram, Statistics
from periodfind_b200 import _native
from periodfind_b200._utils import ensure_float32, prepare_magnitudes, validate_inputs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# ---------------------------------------------------------------- _utils
# Behaviour of periodfind/_utils.py (tests/test_periodfind.py:64-117).

def test_prepare_normalize_range():
    r = prepare_magnitudes([np.array([1, 2, 3], np.float32)], False, True)[0]
    assert r.dtype == np.float32
    assert r.min() >= 0.0 and r.max() <= 1.0


def test_prepare_center():
    r = prepare_magnitudes([np.array([1, 2, 3], np.float32)], True, False)[0]
    assert abs(np.mean(r)) < 1e-6


def test_prepare_passthrough():
    a = np.array([1, 2, 3], np.float32)
    assert prepare_magnitudes([a], False, False)[0] is a


def test_prepare_conflict_warns_and_centers():
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        r = prepare_magnitudes([np.array([1, 2, 3], np.float32)], True, True)[0]
    assert any(issubclass(x.category, RuntimeWarning) for x in w)
    assert abs(np.mean(r)) < 1e-6


def test_validate_inputs():
    validate_inputs([np.zeros(2)], [np.zeros(2)])
    with pytest.raises(ValueError, match="same number of light curves"):
        validate_inputs([np.zeros(2), np.zeros(2)], [np.zeros(2)])
    with pytest.raises(ValueError, match="different lengths"):
        validate_inputs([np.zeros(3)], [np.zeros(2)])


def test_ensure_float32():
    ensure_float32([np.zeros(2, np.float32)], "x")
    with pytest.raises(TypeError, match="float64.*expected float32"):
        ensure_float32([np.zeros(2)], "x")


# ------------------------------------------------- Statistics / Periodogram

def test_statistics_significance():
    s = Statistics([1.0, 0.0], 5.0, 2.0, 1.5, 2.5, 0.5)
    assert s.significance == pytest.approx(2.0)
    s.significance_type = "madmedian"
    assert s.significance == pytest.approx(5.0)
    s.significance_type = "nope"
    with pytest.raises(NotImplementedError):
        _ = s.significance
    assert "Statistics(params=" in repr(s)


def test_statistics_from_data_max_min_multi():
    data = np.array([[1.0], [5.0], [3.0], [0.5]], np.float32)
    params = [np.array([10, 20, 30, 40], np.float32), np.array([0.0], np.float32)]
    s = Statistics.statistics_from_data(data, params, True)
    assert s.params[0] == 20 and s.value == 5.0
    s = Statistics.statistics_from_data(data, params, False)
    assert s.params[0] == 40
    lst = Statistics.statistics_from_data(data, params, True, n=3)
    assert [x.value for x in lst] == [5.0, 3.0, 1.0]
    assert lst[0].mean == pytest.approx(np.mean(data))
    assert lst[0].median == pytest.approx(np.median(data))


def test_periodogram_best_params():
    data = np.array([[1.0], [5.0], [3.0]], np.float32)
    params = [np.array([1, 2, 3], np.float32), np.array([0.0], np.float32)]
    pg = Periodogram(data, params, True)
    assert "use_max=True" in repr(pg)
    b = pg.best_params()
    assert b.params[0] == 2
    assert pg.mean is not None and pg.mad is not None
    assert Periodogram(data, params, False).best_params().params[0] == 1


# -------------------------------------------------------------- C ABI


def _declared_symbols():
    with open(os.path.join(ROOT, "include", "pf.h")) as fh:
        text = fh.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pf_[a-z0-9_]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert _declared_symbols() == sorted(_native.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_native.LIB_PATH)
    for name in _declared_symbols():
        assert hasattr(lib, name), name


def test_no_oracle_in_product_path():
    """The product package never imports the test oracle."""
    pkg = os.path.join(ROOT, "periodfind_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".inc", ".pyx", ".pxi", ".pxd")):
                with open(os.path.join(dirpath, f)) as fh:
                    src = fh.read()
                assert "oracle" not in src.lower().replace("oracle/", ""), f


# ----------------------------------------- GPU classes: checks before device work

def _gpu_classes():
    from periodfind_b200 import gpu

    return gpu


def test_invalid_output_raises_before_device_work():
    gpu = _gpu_classes()
    t = np.arange(5, dtype=np.float32)
    with pytest.raises(NotImplementedError):
        gpu.ConditionalEntropy().calc([t], [t], np.ones(3, np.float32), np.zeros(1, np.float32),
                                      output="invalid")


def test_float64_inputs_raise():
    gpu = _gpu_classes()
    t = np.arange(3, dtype=np.float64)
    with pytest.raises(TypeError, match="expected float32"):
        gpu.ConditionalEntropy().calc([t], [t], np.ones(3, np.float32), np.zeros(1, np.float32))


def test_mismatched_inputs_raise():
    gpu = _gpu_classes()
    t = np.arange(3, dtype=np.float32)
    with pytest.raises(ValueError):
        gpu.AOV().calc([t, t], [t], np.ones(3, np.float32), np.zeros(1, np.float32))


def test_grid_type_checks():
    gpu = _gpu_classes()
    t = np.arange(3, dtype=np.float32)
    with pytest.raises(ValueError, match="dtype mismatch"):
        gpu.LombScargle().calc([t], [t], np.ones(3), np.zeros(1, np.float32))
    with pytest.raises(TypeError):
        gpu.LombScargle().calc([t], [t], [1.0, 2.0], np.zeros(1, np.float32))


def test_mode_and_semantics_validation():
    gpu = _gpu_classes()
    with pytest.raises(ValueError):
        gpu.AOV(mode="fast")
    with pytest.raises(ValueError):
        gpu.AOV(semantics="rust")
    assert gpu.AOV(mode="plain", semantics="cpu")._flags == _native.PF_SEM_CPU
    assert gpu.LombScargle(fold="df")._flags & _native.PF_FOLD_DF


def test_native_normalisation_matches_numpy_bit_for_bit():
    """prepare_magnitudes(normalize=True) runs in the native library for
    float32 batches; every value equals numpy's evaluation of the reference
    expression, including NaN / inf / constant / single-point / tiny curves."""
    import warnings

    from periodfind_b200._utils import prepare_magnitudes

    rng = np.random.default_rng(12)
    ms = [rng.normal(15, 0.3, int(n)).astype(np.float32) for n in rng.integers(1, 3000, 300)]
    ms[3][5] = np.nan
    ms[7][:] = 2.0
    ms[9][2] = np.inf
    ms[11] = np.array([1.0], np.float32)
    ms[13] = (rng.normal(size=777) * 1e-30).astype(np.float32)
    got = prepare_magnitudes(ms, False, True)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        want = [((m - np.min(m)) / (np.max(m) - np.min(m))) * 0.999 + 5e-4 for m in ms]
    for g, w in zip(got, want):
        assert g.dtype == w.dtype == np.float32
        np.testing.assert_array_equal(g, w)
    # an empty curve keeps numpy's error
    with pytest.raises(ValueError):
        prepare_magnitudes([np.zeros(0, np.float32)], False, True)


def test_native_centring_matches_numpy_bit_for_bit():
    """prepare_magnitudes(center=True) runs in the native library
    (pf_center_mags, numpy's pairwise float32 sum) for float32 batches;
    every value equals m - np.mean(m), across the pairwise sum's block
    boundaries (7/8/9, 127/128/129 points and longer splits) and with
    NaN, inf, constant and single-point curves."""
    import warnings

    from periodfind_b200._utils import prepare_magnitudes

    rng = np.random.default_rng(13)
    lens = [1, 2, 7, 8, 9, 15, 16, 17, 127, 128, 129, 255, 256, 257, 1023, 1024, 1025, 4097,
            20000, 65537] + [int(n) for n in rng.integers(1, 3000, 200)]
    ms = [(15 + rng.normal(0, 1, n) * rng.uniform(0.01, 3)).astype(np.float32) for n in lens]
    ms[30][5] = np.nan
    ms[31][:] = 7.25
    ms[32][2] = np.inf
    ms[33] = (rng.normal(size=777) * 1e-30).astype(np.float32)
    got = prepare_magnitudes(ms, True, False)
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        want = [m - np.mean(m) for m in ms]
    for g, w in zip(got, want):
        assert g.dtype == w.dtype == np.float32
        np.testing.assert_array_equal(g, w)
    # an empty curve keeps numpy's behaviour (NaN mean, a warning)
    with pytest.warns(RuntimeWarning):
        out = prepare_magnitudes([np.zeros(0, np.float32), np.ones(3, np.float32)], True, False)
    assert out[0].size == 0 and np.array_equal(out[1], np.zeros(3, np.float32))


def test_result_building_restores_collector_state():
    """Result objects are built with the cyclic collector paused; its state
    afterwards is the caller's, enabled or disabled, and the results are
    the reference's (periodfind/cpu/__init__.py:46-70: a curve's list stops
    at its first -1)."""
    import gc

    from periodfind_b200.gpu import unravel_peaks

    periods = np.array([1.0, 2.0, 3.0], np.float32)
    pdts = np.array([0.0, 0.5], np.float32)
    idx = np.array([[5, 0, -1], [2, 3, 4]], np.int64)
    val = np.array([[0.5, 0.25, 0.0], [1.0, 2.0, 3.0]], np.float32)
    assert gc.isenabled()
    out = unravel_peaks(idx, val, periods, pdts, 3)
    assert gc.isenabled()
    assert [len(r) for r in out] == [2, 3]
    assert out[0][0].params == [3.0, 0.5] and out[0][0].value == 0.5
    assert out[1][2].params == [3.0, 0.0] and out[1][2].value == 3.0
    gc.disable()
    try:
        unravel_peaks(idx, val, periods, pdts, 3)
        assert not gc.isenabled()
    finally:
        gc.enable()


def test_curve_pointers_address_the_curves():
    """CurveBatch's per-curve pointers address each curve's float32 data,
    whether short curves are gathered into one buffer, long ones are used in
    place, or the magnitudes come from the batch normalisation (a list whose
    pointers are precomputed, dropped when the list is changed)."""
    from periodfind_b200 import _native as nat
    from periodfind_b200._utils import prepare_magnitudes

    def read(p, n):
        return np.ctypeslib.as_array((ctypes.c_float * n).from_address(int(p)))

    rng = np.random.default_rng(5)
    for sizes in ([5, 700, 1, 64], [3000, 5000, 2500]):
        ts = [rng.uniform(0, 100, k).astype(np.float32) for k in sizes]
        ms = [rng.normal(15, 0.3, k).astype(np.float64) for k in sizes]
        b = nat.CurveBatch(ts, ms)
        assert b.lengths.tolist() == sizes
        for c, k in enumerate(sizes):
            np.testing.assert_array_equal(read(b.tptr[c], k), ts[c])
            np.testing.assert_array_equal(read(b.mptr[c], k), ms[c].astype(np.float32))
        norm = prepare_magnitudes([m.astype(np.float32) for m in ms], False, True)
        sub = norm[1:]
        bn = nat.CurveBatch(ts[1:], sub)
        assert bn.mptr is sub.ptrs
        for c in range(len(sizes) - 1):
            np.testing.assert_array_equal(read(bn.mptr[c], sizes[c + 1]), norm[c + 1])
        norm[0] = norm[0].copy()
        assert norm.ptrs is None
        bc = nat.CurveBatch(ts, norm)
        np.testing.assert_array_equal(read(bc.mptr[0], sizes[0]), norm[0])
    # 1-D contiguous float32 arrays are addressed in place (the compiled
    # helper reads their addresses); a strided view is not, and takes the
    # converting path.
    ts32 = [rng.uniform(0, 100, k).astype(np.float32) for k in (7, 300)]
    ms32 = [rng.normal(15, 0.3, k).astype(np.float32) for k in (7, 300)]
    b = nat.CurveBatch(ts32, ms32)
    assert b.lengths.tolist() == [7, 300]
    assert [int(p) for p in b.tptr] == [a.ctypes.data for a in ts32]
    assert [int(p) for p in b.mptr] == [a.ctypes.data for a in ms32]
    strided = [np.arange(20, dtype=np.float32)[::2], ms32[1][:10]]
    b = nat.CurveBatch([ts32[1][:10], ts32[1][10:20]], strided)
    for c in range(2):
        np.testing.assert_array_equal(read(b.mptr[c], 10), strided[c])
    with pytest.raises(ValueError):
        nat.CurveBatch([np.zeros(3, np.float32)], [np.zeros(4, np.float32)])


def test_chunked_peaks_pipeline_order_and_error_cleanup(monkeypatch):
    """The 'peaks' pipeline (gpu._Periodogram._chunked_peaks) against a fake
    context: chunks cover the curves in order, at most two calls are
    pending when one is collected, results come back in curve order, and a
    failing call still has every queued call collected, so the context is
    left with nothing pending."""
    import threading

    from periodfind_b200 import gpu

    class FakeLib:
        def __init__(self, ctx):
            self.ctx = ctx

        def pf_wait(self, handle):
            assert self.ctx.pending > 0
            self.ctx.pending -= 1
            return 0

    class FakeCtx:
        lock = threading.Lock()
        handle = None

        def __init__(self):
            self.pending = 0
            self.max_pending = 0
            self.lib = FakeLib(self)

        def check(self, rc):
            if rc != 0:
                raise RuntimeError(f"native call failed: {rc}")
            return rc

    ctx = FakeCtx()
    monkeypatch.setattr(gpu.nat, "default_context", lambda device=0: ctx)
    P = np.linspace(1.0, 2.0, 5).astype(np.float32)
    D = np.zeros(1, np.float32)
    chunks = []

    def issue(c, a, e, idx, val, fail_at=None):
        if fail_at is not None and len(chunks) == fail_at:
            return -2
        chunks.append((a, e))
        c.pending += 1
        c.max_pending = max(c.max_pending, c.pending)
        idx[:, 0] = np.arange(a, e) % len(P)  # peak k of curve i at cell i mod 5
        val[:, 0] = np.arange(a, e)
        return 0

    obj = gpu.AOV()
    res = obj._chunked_peaks(200, P, D, 1, issue)
    assert chunks[0][0] == 0 and chunks[-1][1] == 200
    assert all(x[1] == y[0] for x, y in zip(chunks, chunks[1:]))
    assert ctx.pending == 0 and ctx.max_pending == 2
    assert [r[0].value for r in res] == list(range(200))
    assert [r[0].params[0] for r in res] == [P[i % 5] for i in range(200)]
    chunks.clear()
    with pytest.raises(RuntimeError):
        obj._chunked_peaks(200, P, D, 1, lambda *a: issue(*a, fail_at=3))
    assert len(chunks) == 3 and ctx.pending == 0
    with pytest.raises(ValueError):
        obj._chunked_peaks(200, P, D, -1, issue)


def test_dropin_declarations_are_in_the_header():
    """Every C function the drop-in Cython modules declare
    (periodfind_b200/dropin/pf_abi.pxd) is declared in include/pf.h."""
    with open(os.path.join(ROOT, "periodfind_b200", "dropin", "pf_abi.pxd")) as fh:
        pxd = set(re.findall(r"\b(pf_[a-z0-9_]+)\s*\(", fh.read()))
    assert pxd and pxd <= set(_declared_symbols())
