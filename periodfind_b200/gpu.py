"""GPU periodogram classes: drop-ins for periodfind.gpu.{ConditionalEntropy,
AOV, LombScargle} (periodfind/ce.pyx:41-209, aov.pyx:38-192, ls.pyx:37-176).

Constructor arguments and `calc()` keep the reference's names, defaults and
errors.  `calc()` takes the superset signature of the reference's CPU
classes (periodfind/cpu/__init__.py:73-397): `output` may also be 'peaks'
(with `n_peaks`, `min_distance`), and `errs` is accepted and ignored, as
CE, AOV and LS do not use uncertainties.

Keyword-only additions select the implementation:
  mode       'chosen' (default) or 'plain' (the reference's fold, op for op)
  semantics  'cuda' (default: the reference CUDA build's arithmetic) or
             'cpu' (the reference CPU path's IEEE arithmetic)
  reference_stats  (CE, AOV) True: the chosen form computes the statistic
             from its bins with the reference's operation sequence, so its
             values equal the plain form's exactly when the bins do
"""

from __future__ import annotations

import numpy as np

from . import _host
from . import _native as nat
from ._utils import ensure_float32, gc_paused, prepare_magnitudes, validate_inputs
from .results import Periodogram, Statistics

N_PEAKS_DEFAULT = 32
MIN_DISTANCE_DEFAULT = 1
_OUTPUTS = ("stats", "periodogram", "peaks")


def _mode_flags(mode: str, semantics: str, fold: str | None = None,
                reference_stats: bool = False) -> int:
    if mode not in ("chosen", "plain"):
        raise ValueError(f"mode must be 'chosen' or 'plain', got {mode!r}")
    if semantics not in ("cuda", "cpu"):
        raise ValueError(f"semantics must be 'cuda' or 'cpu', got {semantics!r}")
    f = nat.PF_MODE_CHOSEN if mode == "chosen" else nat.PF_MODE_PLAIN
    if semantics == "cpu":
        f |= nat.PF_SEM_CPU
    if fold == "df":
        f |= nat.PF_FOLD_DF
    elif fold == "f32":
        f |= nat.PF_FOLD_F32
    elif fold == "exact":
        f |= nat.PF_FOLD_EXACT
    elif fold not in (None, "ref"):
        raise ValueError(f"unknown fold {fold!r}")
    if reference_stats:
        f |= nat.PF_REF_STATS
    return f


def _grid(a, name):
    # The reference types these as 1-D float32 ndarrays (ce.pyx:89-90).
    if not isinstance(a, np.ndarray):
        raise TypeError(f"Argument '{name}' has incorrect type (expected numpy.ndarray, "
                        f"got {type(a).__name__})")
    if a.ndim != 1:
        raise ValueError(f"Buffer has wrong number of dimensions (expected 1, got {a.ndim})")
    if a.dtype != np.float32:
        raise ValueError(f"Buffer dtype mismatch, expected 'float32_t' but got '{a.dtype}'")
    return np.ascontiguousarray(a)


def _fused_prep(mags, center, normalize, known_ok=False):
    """(magnitudes to pass, extra mode bits).  For float32 1-D curves that
    are all non-empty the native packing prepares the magnitudes itself
    (PF_HOST_CENTER / PF_HOST_NORMALIZE: numpy's values, no separate pass
    or copy); anything else is prepared here as the reference does.  The
    centre / normalise conflict is settled by the caller.  known_ok: the
    batch was already found to have that form."""
    if not (center or normalize):
        return mags, 0
    if known_ok or all(isinstance(m, np.ndarray) and m.ndim == 1 and m.size
                       and m.dtype == np.float32 for m in mags):
        return mags, (nat.PF_HOST_CENTER if center else nat.PF_HOST_NORMALIZE)
    return prepare_magnitudes(mags, center, normalize), 0


def unravel_peaks(peak_indices, peak_values, periods, period_dts, n_peaks):
    """Flat peak indices -> list (per curve) of lists of Statistics, stopping
    at the first -1 (periodfind/cpu/__init__.py:46-70)."""
    n_pdts = len(period_dts)
    idx = np.asarray(peak_indices, dtype=np.int64)[:, :n_peaks]
    valid = idx >= 0
    # Each curve's list stops at its first -1.
    count = np.where(valid.all(axis=1), idx.shape[1], np.argmin(valid, axis=1)).tolist()
    safe = np.where(valid, idx, 0)
    per = np.asarray(periods)[safe // n_pdts].astype(np.float64).tolist()
    pdt = np.asarray(period_dts)[safe % n_pdts].astype(np.float64).tolist()
    val = np.asarray(peak_values)[:, :n_peaks].astype(np.float64).tolist()
    with gc_paused():
        return [[Statistics([pr[k], dr[k]], vr[k], 0.0, 1.0, 0.0, 1.0) for k in range(cnt)]
                for pr, dr, vr, cnt in zip(per, pdt, val, count)]


class _Periodogram:
    _use_max = True
    _normalize_default = False
    _center_default = False

    def __init__(self, *, mode="chosen", semantics="cuda", device=0):
        self.mode = mode
        self.semantics = semantics
        self.device = device
        self._flags = _mode_flags(mode, semantics, getattr(self, "_fold", None),
                                  getattr(self, "_reference_stats", False))

    # -- native calls, implemented per algorithm
    def _native_pgram(self, ctx, b, periods, pdts, out, extra=0):
        raise NotImplementedError

    def _native_peaks(self, ctx, b, periods, pdts, n_peaks, min_distance, idx, val, extra=0):
        raise NotImplementedError

    def periodograms(self, times, mags, periods, period_dts, _extra=0):
        """Raw [n_curves, n_periods, n_pdts] float32 array for prepared mags."""
        ctx = nat.default_context(self.device)
        b = nat.CurveBatch(times, mags)
        out = np.empty((b.n, len(periods), len(period_dts)), dtype=np.float32)
        with ctx.lock:
            ctx.check(self._native_pgram(ctx, b, periods, period_dts, out, _extra))
        return out

    def bin_counts(self, times, mags, periods, period_dts):
        """(periodogram float32 [n_curves, n_periods, n_pdts], raw bin counts
        uint32 [n_curves, n_periods, n_pdts, bins]) for prepared magnitudes,
        from this object's kernels (pf_bin_counts); bins = n_phase * n_mag
        (CE, phase-major) or n_phase (AOV).  The counterpart of the
        reference's ConditionalEntropy::FoldAndBin / AOV::FoldAndBin
        (periodfind/cuda/ce.h:194, aov.h:132), for occupancy checks.  CE and
        AOV only."""
        if not hasattr(self, "_bin_args"):
            raise NotImplementedError("bin counts exist for ConditionalEntropy and AOV only")
        algo, n_phase, n_mag, po, mo = self._bin_args()
        periods = _grid(periods, "periods")
        period_dts = _grid(period_dts, "period_dts")
        ctx = nat.default_context(self.device)
        b = nat.CurveBatch(times, mags)
        nb = n_phase * n_mag if algo == nat.PF_ALGO_CE else n_phase
        out = np.empty((b.n, len(periods), len(period_dts)), dtype=np.float32)
        counts = np.zeros((b.n, len(periods), len(period_dts), nb), dtype=np.uint32)
        with ctx.lock:
            ctx.check(ctx.lib.pf_bin_counts(ctx.handle, algo, *b.args(), nat.ptr(periods),
                                            len(periods), nat.ptr(period_dts), len(period_dts),
                                            n_phase, n_mag, po, mo, self._flags, nat.ptr(out),
                                            nat.ptr(counts)))
        return out, counts

    def periodograms_device(self, t, m, offsets, periods, period_dts, normalize=None,
                            center=None):
        """Periodograms of curves already on the GPU, left on the GPU.

        t, m: contiguous 1-D float32 CUDA tensors on this object's device
        holding the curves back to back (curve c is [offsets[c],
        offsets[c+1])); offsets: n_curves + 1 int64 values (host).  The
        magnitudes are prepared on the device as calc() prepares them (CE
        normalises, LS centres; `normalize` / `center` override), with
        numpy's values bit for bit.  Returns a float32 CUDA tensor [n_curves,
        n_periods, n_pdts] on the current stream (DLPack through torch).  No
        counterpart in the reference, whose results always come back to the
        host."""
        import torch

        if normalize is None:
            normalize = self._normalize_default
        if center is None:
            center = self._center_default
        if center and normalize:  # the reference's conflict warning, then centre
            prepare_magnitudes([], center, normalize)
            normalize = False
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        if off.ndim != 1 or len(off) < 1:
            raise ValueError("offsets must be a 1-D array of n_curves + 1 values")
        n = len(off) - 1
        for name, a in (("t", t), ("m", m)):
            if not (torch.is_tensor(a) and a.is_cuda and a.dtype == torch.float32
                    and a.dim() == 1 and a.is_contiguous()):
                raise TypeError(f"{name} must be a contiguous 1-D float32 CUDA tensor")
            if a.device.index != self.device:
                raise ValueError(f"{name} is on cuda:{a.device.index}, not cuda:{self.device}")
        if t.numel() != m.numel() or off[0] < 0 or off[-1] > t.numel() or np.any(np.diff(off) < 0):
            raise ValueError("offsets must be non-decreasing and within the tensors")
        periods = _grid(periods, "periods")
        period_dts = _grid(period_dts, "period_dts")
        dev = t.device
        stream = torch.cuda.current_stream(dev).cuda_stream
        out = torch.empty((n, len(periods), len(period_dts)), dtype=torch.float32, device=dev)
        if n == 0:
            return out
        kind = nat.PF_PREP_CENTER if center else (nat.PF_PREP_NORMALIZE if normalize else 0)
        ctx = nat.default_context(self.device)
        d_p = torch.from_numpy(periods).to(dev)
        d_d = torch.from_numpy(period_dts).to(dev)
        mp = m
        with ctx.lock:
            if kind:
                mp = torch.empty_like(m)
                ctx.check(ctx.lib.pf_prepare_mags_dev(ctx.handle, m.data_ptr(), off.ctypes.data,
                                                      n, kind, mp.data_ptr(), stream))
            ctx.check(self._native_dev(ctx, t.data_ptr(), mp.data_ptr(), off, n,
                                       d_p.data_ptr(), len(periods), d_d.data_ptr(),
                                       len(period_dts), out.data_ptr(), stream))
        return out

    def _native_dev(self, ctx, d_t, d_m, off, n, d_p, n_per, d_d, n_pdt, d_out, stream):
        raise NotImplementedError

    def peaks(self, times, mags, periods, period_dts, n_peaks=N_PEAKS_DEFAULT,
              min_distance=MIN_DISTANCE_DEFAULT):
        """(indices int64 [n_curves, n_peaks] with -1 padding, values float32)."""
        ctx = nat.default_context(self.device)
        b = nat.CurveBatch(times, mags)
        n_peaks = int(n_peaks)
        if n_peaks < 0:
            raise ValueError("n_peaks must be >= 0")
        idx = np.full((b.n, n_peaks), -1, dtype=np.int64)
        val = np.zeros((b.n, n_peaks), dtype=np.float32)
        with ctx.lock:
            ctx.check(self._native_peaks(ctx, b, periods, period_dts, n_peaks,
                                         int(min_distance), idx, val))
        return idx, val

    # Chunk boundaries of a pipelined 'peaks' batch (fractions of its
    # curves).  The first chunk is small so that the GPU starts early, and
    # so is the last, whose result building nothing overlaps.
    _CHUNK_EDGES = (0.0, 0.1, 0.37, 0.64, 0.9, 1.0)

    @staticmethod
    def _pipelined(times, periods, period_dts):
        """Whether a 'peaks' batch is large enough to run in chunks."""
        points = sum(len(t) for t in times)
        return len(times) >= 64 and points * len(periods) * len(period_dts) >= 2e10

    def _chunked_peaks(self, n, periods, period_dts, n_peaks, issue):
        """'peaks' output of n curves as a few consecutive chunks in a
        pipeline.  issue(ctx, a, e, idx, val) makes the native peak call for
        curves [a, e) with PF_ASYNC: it packs and queues the chunk and
        returns, so the next chunk is prepared, packed and queued while the
        GPU runs this one, and a chunk's result objects are built while the
        GPU runs the next.  Results are identical to one call."""
        n_peaks = int(n_peaks)
        if n_peaks < 0:
            raise ValueError("n_peaks must be >= 0")
        ctx = nat.default_context(self.device)
        bounds = [round(n * f) for f in self._CHUNK_EDGES]
        n_chunks = len(bounds) - 1
        outs = []  # (indices, values) of each queued chunk, alive until collected
        res = []
        with ctx.lock:
            def queue(k):
                a, e = bounds[k], bounds[k + 1]
                idx = np.full((e - a, n_peaks), -1, dtype=np.int64)
                val = np.zeros((e - a, n_peaks), dtype=np.float32)
                ctx.check(issue(ctx, a, e, idx, val))
                outs.append((idx, val))

            collected = 0
            try:
                queue(0)
                for k in range(n_chunks):
                    if k + 1 < n_chunks:
                        queue(k + 1)
                    collected += 1
                    ctx.check(ctx.lib.pf_wait(ctx.handle))
                    idx, val = outs[k]
                    res.extend(unravel_peaks(idx, val, periods, period_dts, n_peaks))
            finally:
                # After an error, collect what is still queued so that the
                # context is left with nothing pending.
                for _ in range(len(outs) - collected):
                    ctx.lib.pf_wait(ctx.handle)
        return res

    def _peaks_overlapped(self, times, mags, periods, period_dts, n_peaks, min_distance,
                          center=False, normalize=False):
        """'peaks' output, with the magnitudes prepared here (centre or
        normalise) per chunk of a pipelined batch (_chunked_peaks)."""
        if not self._pipelined(times, periods, period_dts):
            mags = prepare_magnitudes(mags, center, normalize)
            idx, val = self.peaks(times, mags, periods, period_dts, n_peaks, min_distance)
            return unravel_peaks(idx, val, periods, period_dts, n_peaks)

        def issue(ctx, a, e, idx, val):
            m, extra = _fused_prep(mags[a:e], center, normalize)
            b = nat.CurveBatch(times[a:e], m)
            return self._native_peaks(ctx, b, periods, period_dts, idx.shape[1],
                                      int(min_distance), idx, val, nat.PF_ASYNC | extra)

        return self._chunked_peaks(len(times), periods, period_dts, n_peaks, issue)

    def _stats_on_device(self, times, mags, periods, period_dts, n_stats, significance_type,
                         extra=0):
        """The 'stats' output with the statistics computed on the device
        (identical to numpy's); None where the device path does not apply."""
        ctx = nat.default_context(self.device)
        b = nat.CurveBatch(times, mags)
        st = np.empty((b.n, 4), dtype=np.float32)
        idx = np.empty((b.n, n_stats), dtype=np.int64)
        val = np.empty((b.n, n_stats), dtype=np.float32)
        with ctx.lock:
            rc = self._native_stats(ctx, b, periods, period_dts, n_stats, st, idx, val, extra)
            if rc == nat.PF_EUNSUPPORTED:
                return None
            ctx.check(rc)
        return _stats_from_device(st, idx, val, periods, period_dts, n_stats, significance_type)

    def calc(self, times, mags, periods, period_dts, output="stats", normalize=None,
             center=None, n_stats=1, significance_type="stdmean", n_peaks=N_PEAKS_DEFAULT,
             min_distance=MIN_DISTANCE_DEFAULT, errs=None):
        """Compute the periodogram of every light curve.

        Returns a list of Statistics (output='stats'; lists of them when
        n_stats > 1), a list of Periodogram (output='periodogram'), or a list
        of lists of Statistics for the top peaks (output='peaks').
        """
        if normalize is None:
            normalize = self._normalize_default
        if center is None:
            center = self._center_default
        if output not in _OUTPUTS:
            raise NotImplementedError(
                f'Output type "{output}" is not implemented. '
                f'Use "stats", "periodogram", or "peaks".')
        # A batch already in the native calls' form (float32 1-D contiguous
        # curves, lengths pairing up) needs none of the per-array checks;
        # anything else gets them, with the reference's exceptions.
        form = _host.curve_check(times, mags)
        if not form:
            validate_inputs(times, mags)
            ensure_float32(times, "times")
            ensure_float32(mags, "mags")
        periods = _grid(periods, "periods")
        period_dts = _grid(period_dts, "period_dts")
        if output == "peaks":
            # The magnitudes are prepared chunk by chunk inside the pipeline;
            # the centre / normalise conflict warns once, here.
            if center and normalize:
                prepare_magnitudes([], center, normalize)
                normalize = False
            return self._peaks_overlapped(times, mags, periods, period_dts, int(n_peaks),
                                          min_distance, center, normalize)
        if center and normalize:  # the reference's conflict warning, then centre
            prepare_magnitudes([], center, normalize)
            normalize = False
        mags_use, extra = _fused_prep(mags, center, normalize, known_ok=form == 2)

        if (output == "stats" and 1 <= int(n_stats) < len(periods) * len(period_dts)
                and (not self._use_max or len(period_dts) == 1)):
            res = self._stats_on_device(times, mags_use, periods, period_dts, int(n_stats),
                                        significance_type, extra)
            if res is not None:
                return res

        data = self.periodograms(times, mags_use, periods, period_dts, extra)
        with gc_paused():
            if output == "stats":
                return [Statistics.statistics_from_data(
                    data[i], [periods, period_dts], self._use_max, n=n_stats,
                    significance_type=significance_type) for i in range(len(times))]
            return [Periodogram(d, [periods, period_dts], self._use_max) for d in data]


def _stats_from_device(st, idx, val, periods, period_dts, n_stats, significance_type):
    """Statistics objects from the device statistics, typed as the reference
    builds them from numpy (float32 scalars), best first."""
    n_pdt = len(period_dts)
    # numpy float32 scalars throughout, as the reference's numpy statistics
    # hold them; list() makes a row's scalars in one call.
    k = idx.shape[1]
    per = list(np.asarray(periods)[idx // n_pdt].ravel())
    pdt = list(np.asarray(period_dts)[idx % n_pdt].ravel())
    vals = list(np.asarray(val).ravel())
    summ = list(np.asarray(st).ravel())
    out = []
    with gc_paused():
        for c in range(st.shape[0]):
            mean, std, median, mad = summ[4 * c:4 * c + 4]
            best = [Statistics([per[c * k + j], pdt[c * k + j]], vals[c * k + j], mean, std,
                               median, mad, significance_type) for j in range(k)]
            out.append(best[0] if n_stats == 1 else best)
    return out


class ConditionalEntropy(_Periodogram):
    """Conditional Entropy periodogram (minimum is best).

    n_phase x n_mag histogram of (folded phase, normalised magnitude);
    phase_bin_extent / mag_bin_extent widen each entry over neighbouring
    bins with wrap-around (periodfind/ce.pyx:41-80).
    """

    _use_max = False
    _normalize_default = True

    def __init__(self, n_phase=10, n_mag=10, phase_bin_extent=1, mag_bin_extent=1, *,
                 mode="chosen", semantics="cuda", device=0, reference_stats=False):
        self._reference_stats = bool(reference_stats)
        super().__init__(mode=mode, semantics=semantics, device=device)
        self.n_phase = int(n_phase)
        self.n_mag = int(n_mag)
        self.phase_bin_extent = int(phase_bin_extent)
        self.mag_bin_extent = int(mag_bin_extent)

    def _bin_args(self):
        return (nat.PF_ALGO_CE, self.n_phase, self.n_mag, self.phase_bin_extent,
                self.mag_bin_extent)

    def _native_pgram(self, ctx, b, periods, pdts, out, extra=0):
        return ctx.lib.pf_ce(ctx.handle, *b.args(), nat.ptr(periods), len(periods),
                             nat.ptr(pdts), len(pdts), self.n_phase, self.n_mag,
                             self.phase_bin_extent, self.mag_bin_extent, self._flags | extra,
                             nat.ptr(out))

    def _native_stats(self, ctx, b, periods, pdts, n_top, st, idx, val, extra=0):
        return ctx.lib.pf_ce_stats(ctx.handle, *b.args(), nat.ptr(periods), len(periods),
                                   nat.ptr(pdts), len(pdts), self.n_phase, self.n_mag,
                                   self.phase_bin_extent, self.mag_bin_extent, n_top,
                                   self._flags | extra, nat.ptr(st), nat.ptr(idx),
                                   nat.ptr(val))

    def _native_dev(self, ctx, d_t, d_m, off, n, d_p, n_per, d_d, n_pdt, d_out, stream):
        return ctx.lib.pf_ce_dev(ctx.handle, d_t, d_m, off.ctypes.data, n, d_p, n_per, d_d,
                                 n_pdt, self.n_phase, self.n_mag, self.phase_bin_extent,
                                 self.mag_bin_extent, self._flags, d_out, stream)

    def _native_peaks(self, ctx, b, periods, pdts, n_peaks, min_distance, idx, val, extra=0):
        return ctx.lib.pf_ce_peaks(ctx.handle, *b.args(), nat.ptr(periods), len(periods),
                                   nat.ptr(pdts), len(pdts), self.n_phase, self.n_mag,
                                   self.phase_bin_extent, self.mag_bin_extent, n_peaks,
                                   min_distance, self._flags | extra, nat.ptr(idx),
                                   nat.ptr(val))


class AOV(_Periodogram):
    """Analysis-of-Variance periodogram (maximum is best)
    (periodfind/aov.pyx:38-67)."""

    _use_max = True

    def __init__(self, n_phase=10, phase_bin_extent=1, *, mode="chosen", semantics="cuda",
                 device=0, reference_stats=False):
        self._reference_stats = bool(reference_stats)
        super().__init__(mode=mode, semantics=semantics, device=device)
        self.n_phase = int(n_phase)
        self.phase_bin_extent = int(phase_bin_extent)

    def _bin_args(self):
        return (nat.PF_ALGO_AOV, self.n_phase, 1, self.phase_bin_extent, 1)

    def _native_pgram(self, ctx, b, periods, pdts, out, extra=0):
        return ctx.lib.pf_aov(ctx.handle, *b.args(), nat.ptr(periods), len(periods),
                              nat.ptr(pdts), len(pdts), self.n_phase, self.phase_bin_extent,
                              self._flags | extra, nat.ptr(out))

    def _native_stats(self, ctx, b, periods, pdts, n_top, st, idx, val, extra=0):
        return ctx.lib.pf_aov_stats(ctx.handle, *b.args(), nat.ptr(periods), len(periods),
                                    nat.ptr(pdts), len(pdts), self.n_phase,
                                    self.phase_bin_extent, n_top, self._flags | extra,
                                    nat.ptr(st), nat.ptr(idx), nat.ptr(val))

    def _native_dev(self, ctx, d_t, d_m, off, n, d_p, n_per, d_d, n_pdt, d_out, stream):
        return ctx.lib.pf_aov_dev(ctx.handle, d_t, d_m, off.ctypes.data, n, d_p, n_per, d_d,
                                  n_pdt, self.n_phase, self.phase_bin_extent, self._flags,
                                  d_out, stream)

    def _native_peaks(self, ctx, b, periods, pdts, n_peaks, min_distance, idx, val, extra=0):
        return ctx.lib.pf_aov_peaks(ctx.handle, *b.args(), nat.ptr(periods), len(periods),
                                    nat.ptr(pdts), len(pdts), self.n_phase,
                                    self.phase_bin_extent, n_peaks, min_distance,
                                    self._flags | extra, nat.ptr(idx), nat.ptr(val))


class LombScargle(_Periodogram):
    """Lomb-Scargle periodogram (maximum is best; magnitudes centred by
    default) (periodfind/ls.pyx:37-62).

    The chosen form folds with a split-precision FP32 phase; fold='exact'
    selects the divide-free exact fold (bit-identical to the plain form),
    fold='f32' the all-FP32 fold (precision studies).
    """

    _use_max = True
    _center_default = True

    def __init__(self, *, mode="chosen", semantics="cuda", device=0, fold=None):
        self._fold = fold
        super().__init__(mode=mode, semantics=semantics, device=device)

    def _native_pgram(self, ctx, b, periods, pdts, out, extra=0):
        return ctx.lib.pf_ls(ctx.handle, *b.args(), nat.ptr(periods), len(periods),
                             nat.ptr(pdts), len(pdts), self._flags | extra, nat.ptr(out))

    def _native_stats(self, ctx, b, periods, pdts, n_top, st, idx, val, extra=0):
        return ctx.lib.pf_ls_stats(ctx.handle, *b.args(), nat.ptr(periods), len(periods),
                                   nat.ptr(pdts), len(pdts), n_top, self._flags | extra,
                                   nat.ptr(st), nat.ptr(idx), nat.ptr(val))

    def _native_dev(self, ctx, d_t, d_m, off, n, d_p, n_per, d_d, n_pdt, d_out, stream):
        return ctx.lib.pf_ls_dev(ctx.handle, d_t, d_m, off.ctypes.data, n, d_p, n_per, d_d,
                                 n_pdt, self._flags, d_out, stream)

    def _native_peaks(self, ctx, b, periods, pdts, n_peaks, min_distance, idx, val, extra=0):
        return ctx.lib.pf_ls_peaks(ctx.handle, *b.args(), nat.ptr(periods), len(periods),
                                   nat.ptr(pdts), len(pdts), n_peaks, min_distance,
                                   self._flags | extra, nat.ptr(idx), nat.ptr(val))

    def periodograms_frequency_grid(self, times, mags, f_min, df, n_freq, trig=None,
                                    center=None):
        """LS power at the trial frequencies f_min + k * df (cycles per time
        unit), k < n_freq, as float32 [n_curves, n_freq]; magnitudes centred
        as calc() centres them.  No counterpart in the reference, whose grid
        is an array of trial periods (pf_ls_fgrid).

        On a uniform frequency grid the phase of a point advances by the same
        angle from one frequency to the next, so the sine and cosine can
        follow the grid by angle-addition rotations instead of one MUFU pair
        per evaluation.  trig: None lets the autotuner pick per curve-length
        class; 'sincos' or 'recurrence' keeps one form.  Chosen form and
        CUDA arithmetic only (fold='exact' for an FP64 phase)."""
        if self.mode != "chosen" or self.semantics != "cuda":
            raise ValueError("a frequency grid needs mode='chosen', semantics='cuda'")
        if trig not in (None, "sincos", "recurrence"):
            raise ValueError(f"trig must be None, 'sincos' or 'recurrence', got {trig!r}")
        if center is None:
            center = self._center_default
        validate_inputs(times, mags)
        ensure_float32(times, "times")
        ensure_float32(mags, "mags")
        mags_use = prepare_magnitudes(mags, center, False)
        flags = self._flags | {None: 0, "sincos": nat.PF_TRIG_SINCOS,
                               "recurrence": nat.PF_TRIG_RECURRENCE}[trig]
        ctx = nat.default_context(self.device)
        b = nat.CurveBatch(times, mags_use)
        out = np.empty((b.n, int(n_freq)), dtype=np.float32)
        with ctx.lock:
            ctx.check(ctx.lib.pf_ls_fgrid(ctx.handle, *b.args(), float(f_min), float(df),
                                          int(n_freq), flags, nat.ptr(out)))
        return out

    def refine_peaks(self, times, mags, periods, peak_indices, n_steps=5, center=None):
        """Refine grid peaks off the trial grid by Newton steps on dP/domega
        (no counterpart in the reference, whose peaks are grid points).

        peak_indices: [n_curves, K] indices into `periods` (-1 = no peak), as
        peaks() returns them for period_dts=[0].  Each peak is refined inside
        the bracket reaching its farther grid neighbour.  Returns (periods
        float64 [n_curves, K], NaN where no peak; powers float32, 0 there).
        """
        import torch

        from . import ls_grad

        if center is None:
            center = self._center_default
        validate_inputs(times, mags)
        ensure_float32(times, "times")
        ensure_float32(mags, "mags")
        mags_use = prepare_magnitudes(mags, center, False)
        grid = np.asarray(_grid(periods, "periods"), dtype=np.float64)
        idx = np.asarray(peak_indices, dtype=np.int64)
        if idx.ndim != 2 or idx.shape[0] != len(times):
            raise ValueError("peak_indices must be [n_curves, K]")
        if np.any(idx >= len(grid)):
            raise ValueError("peak index out of range of periods")
        valid = idx >= 0
        i = np.where(valid, idx, 0)
        w_grid = 2.0 * np.pi / grid
        w0 = w_grid[i]
        hw = np.maximum(np.abs(w_grid[np.maximum(i - 1, 0)] - w0),
                        np.abs(w_grid[np.minimum(i + 1, len(grid) - 1)] - w0))
        lens = np.array([len(t) for t in times], dtype=np.int64)
        off = np.zeros(len(times) + 1, dtype=np.int64)
        np.cumsum(lens, out=off[1:])
        dev = torch.device("cuda", self.device)
        cat = lambda xs: torch.from_numpy(
            np.concatenate(xs) if len(xs) else np.zeros(0, np.float32)).to(dev)
        w, pw = ls_grad.refine_peaks(cat(list(times)), cat(list(mags_use)),
                                     torch.from_numpy(w0).to(dev), torch.from_numpy(hw).to(dev),
                                     off, n_steps)
        w = w.cpu().numpy()
        pw = pw.cpu().numpy()
        return (np.where(valid, 2.0 * np.pi / np.where(valid, w, 1.0), np.nan),
                np.where(valid, pw, np.float32(0.0)).astype(np.float32))


class FPW(_Periodogram):
    """Fast phase-folding weighted (FPW) periodogram (Finkbeiner et al.
    2025), maximum is best (periodfind/fpw.pyx:29-177; the CPU class
    periodfind/cpu/__init__.py:400-521, whose 'peaks' output it also has).

    Per point an inverse variance 1 / err^2 weights the magnitude; per
    phase bin V = sum of weights, Y = sum of weighted magnitudes; the value
    is sum over non-empty bins of Y^2 / (2 V).  `errs` None means unit
    uncertainties; `normalize` and `center` are accepted and unused, as in
    the reference.
    """

    _use_max = True

    def __init__(self, n_bins=10, *, mode="chosen", semantics="cuda", device=0):
        super().__init__(mode=mode, semantics=semantics, device=device)
        self.n_bins = int(n_bins)

    @staticmethod
    def _check_errs(times, errs):
        # periodfind/cpu/__init__.py:466-481.
        if errs is None:
            return None
        ensure_float32(errs, "errs")
        if len(errs) != len(times):
            raise ValueError(
                f"errs must have the same number of arrays as times, "
                f"got {len(errs)} and {len(times)}")
        for i, (e, t) in enumerate(zip(errs, times)):
            if len(e) != len(t):
                raise ValueError(
                    f"errs[{i}] and times[{i}] have different lengths: {len(e)} vs {len(t)}")
        return errs

    # The native calls and the statistic's own arguments after n_bins.
    _pgram_fn, _peaks_fn = "pf_fpw", "pf_fpw_peaks"

    def _stat_args(self):
        return (self.n_bins,)

    def _call(self, ctx, fn, times, mags, errs, periods, pdts, *tail):
        b = nat.CurveBatch(times, mags)
        eptr, keep = (None, None) if errs is None else nat.host_pointers(errs, b.lengths)
        tptr, mptr, lens, n = b.args()
        rc = fn(ctx.handle, tptr, mptr, None if eptr is None else eptr.ctypes.data, lens, n,
                nat.ptr(periods), len(periods), nat.ptr(pdts), len(pdts), *self._stat_args(),
                *tail)
        del keep
        return rc

    def periodograms(self, times, mags, periods, period_dts, errs=None):
        """Raw [n_curves, n_periods, n_pdts] float32 array."""
        ctx = nat.default_context(self.device)
        out = np.empty((len(times), len(periods), len(period_dts)), dtype=np.float32)
        with ctx.lock:
            ctx.check(self._call(ctx, getattr(ctx.lib, self._pgram_fn), times, mags, errs,
                                 periods, period_dts, self._flags, nat.ptr(out)))
        return out

    def peaks(self, times, mags, periods, period_dts, n_peaks=N_PEAKS_DEFAULT,
              min_distance=MIN_DISTANCE_DEFAULT, errs=None):
        """(indices int64 [n_curves, n_peaks] with -1 padding, values float32)."""
        ctx = nat.default_context(self.device)
        n_peaks = int(n_peaks)
        if n_peaks < 0:
            raise ValueError("n_peaks must be >= 0")
        idx = np.full((len(times), n_peaks), -1, dtype=np.int64)
        val = np.zeros((len(times), n_peaks), dtype=np.float32)
        with ctx.lock:
            ctx.check(self._call(ctx, getattr(ctx.lib, self._peaks_fn), times, mags, errs,
                                 periods, period_dts, n_peaks, int(min_distance), self._flags,
                                 nat.ptr(idx), nat.ptr(val)))
        return idx, val

    def calc(self, times, mags, periods, period_dts, errs=None, output="stats",
             normalize=False, center=False, n_stats=1, significance_type="stdmean",
             n_peaks=N_PEAKS_DEFAULT, min_distance=MIN_DISTANCE_DEFAULT):
        """Compute the periodogram of every light curve.

        Returns a list of Statistics (output='stats'; lists of them when
        n_stats > 1), a list of Periodogram (output='periodogram'), or a list
        of lists of Statistics for the top peaks (output='peaks').
        """
        if output not in _OUTPUTS:
            raise NotImplementedError(
                f'Output type "{output}" is not implemented. '
                f'Use "stats", "periodogram", or "peaks".')
        validate_inputs(times, mags)
        ensure_float32(times, "times")
        ensure_float32(mags, "mags")
        errs = self._check_errs(times, errs)
        periods = _grid(periods, "periods")
        period_dts = _grid(period_dts, "period_dts")
        if output == "peaks":
            if not self._pipelined(times, periods, period_dts):
                idx, val = self.peaks(times, mags, periods, period_dts, n_peaks, min_distance,
                                      errs)
                return unravel_peaks(idx, val, periods, period_dts, int(n_peaks))
            fn = self._peaks_fn

            def issue(ctx, a, e, idx, val):
                return self._call(ctx, getattr(ctx.lib, fn), times[a:e], mags[a:e],
                                  None if errs is None else errs[a:e], periods, period_dts,
                                  idx.shape[1], int(min_distance), self._flags | nat.PF_ASYNC,
                                  nat.ptr(idx), nat.ptr(val))

            return self._chunked_peaks(len(times), periods, period_dts, n_peaks, issue)
        data = self.periodograms(times, mags, periods, period_dts, errs)
        with gc_paused():
            if output == "stats":
                return [Statistics.statistics_from_data(
                    data[i], [periods, period_dts], True, n=n_stats,
                    significance_type=significance_type) for i in range(len(times))]
            return [Periodogram(d, [periods, period_dts], True) for d in data]


class BoxLeastSquares(FPW):
    """Box least squares (BLS, Kovacs, Zucker & Mazeh 2002) transit search,
    maximum is best (periodfind/bls.pyx:36-181; the CPU class
    periodfind/cpu/__init__.py:525-640, whose 'peaks' output it also has).

    Per point an inverse variance w = 1 / err^2 weights the magnitude minus
    the curve's weighted mean; the phase bins' sums are searched for the
    window of qmin .. qmax of the period (in bins, wrapping) with the best
    s^2 / (r (W - r)).  `errs` None means unit uncertainties; `normalize`
    and `center` are accepted and unused, as in the reference.
    """

    _pgram_fn, _peaks_fn = "pf_bls", "pf_bls_peaks"

    def __init__(self, n_bins=50, qmin=0.01, qmax=0.5, *, mode="chosen", semantics="cuda",
                 device=0):
        super().__init__(n_bins, mode=mode, semantics=semantics, device=device)
        self.qmin = float(qmin)
        self.qmax = float(qmax)

    def _stat_args(self):
        return (self.n_bins, self.qmin, self.qmax)


def find_top_peaks_batched(data, n_peaks, min_distance, use_max, device=0):
    """Top peaks of precomputed periodograms [n_curves, n_periods, n_pdts]
    (rust/src/lib.rs:508-548), computed on the GPU."""
    d = np.ascontiguousarray(data, dtype=np.float32)
    if d.ndim != 3:
        raise ValueError("data must have shape (n_curves, n_periods, n_pdts)")
    ctx = nat.default_context(device)
    n_peaks = int(n_peaks)
    idx = np.full((d.shape[0], n_peaks), -1, dtype=np.int64)
    val = np.zeros((d.shape[0], n_peaks), dtype=np.float32)
    with ctx.lock:
        ctx.check(ctx.lib.pf_find_peaks(ctx.handle, nat.ptr(d), d.shape[0],
                                        d.shape[1] * d.shape[2], n_peaks, int(min_distance),
                                        int(bool(use_max)), nat.ptr(idx), nat.ptr(val)))
    return idx, val
