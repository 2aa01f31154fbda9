#cython: language_level=3
"""FPW (fast phase-folding weighted) on the B200, in place of periodfind's
fpw.pyx.

Same class, constructor and calc() as periodfind/fpw.pyx:29-177; the
periodograms come from the C ABI of include/pf.h (pf_fpw, pf_fpw_peaks)
instead of the reference's CalcFPWBatched.  `normalize` and `center` are
accepted and unused, as in the reference.  Additions: output='peaks'
(n_peaks, min_distance) and the keyword-only constructor arguments mode
('chosen' or 'plain') and device.
"""

include "_common.pxi"


cdef class FPW:
    """FPW periodogram over n_bins phase bins, points weighted by 1 / err^2
    (unit uncertainties when errs is None).  The maximum is the best
    period."""

    cdef readonly int n_bins, device
    cdef readonly str mode
    cdef int flags

    def __cinit__(self, n_bins=10, *, mode="chosen", device=0):
        self.n_bins = n_bins
        self.mode = mode
        self.flags = _mode_flags(mode)
        self.device = device

    def calc(self,
             list times,
             list mags,
             cnp.ndarray[ndim=1, dtype=cnp.float32_t] periods,
             cnp.ndarray[ndim=1, dtype=cnp.float32_t] period_dts,
             errs=None,
             output="stats",
             normalize=False,
             center=False,
             n_stats=1,
             significance_type='stdmean',
             n_peaks=N_PEAKS_DEFAULT,
             min_distance=MIN_DISTANCE_DEFAULT):
        """FPW of every light curve over the trial periods and period
        derivatives: a list of Statistics (output='stats'), of Periodogram
        ('periodogram'), or of lists of Statistics for the top peaks
        ('peaks')."""
        validate_inputs(times, mags)
        ensure_float32(times, 'times')
        ensure_float32(mags, 'mags')
        errs = _check_errs(times, errs)
        return _calc(ALGO_FPW, (self.n_bins,), self.flags, self.device, times, list(mags),
                     errs, periods, period_dts, output, True, n_stats, significance_type,
                     n_peaks, min_distance)
