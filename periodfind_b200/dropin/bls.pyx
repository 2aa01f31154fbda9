#cython: language_level=3
"""Box least squares on the B200, in place of periodfind's bls.pyx.

Same class, constructor and calc() as periodfind/bls.pyx:36-181; the
periodograms come from the C ABI of include/pf.h (pf_bls, pf_bls_peaks)
instead of the reference's CalcBLSBatched.  `normalize` and `center` are
accepted and unused, as in the reference.  Additions: output='peaks'
(n_peaks, min_distance) and the keyword-only constructor arguments mode
('chosen' or 'plain') and device.
"""

include "_common.pxi"


cdef class BoxLeastSquares:
    """BLS transit search over n_bins phase bins, windows of qmin .. qmax of
    the period, points weighted by 1 / err^2 (unit uncertainties when errs
    is None).  The maximum is the best period."""

    cdef readonly int n_bins, device
    cdef readonly float qmin, qmax
    cdef readonly str mode
    cdef int flags

    def __cinit__(self, n_bins=50, qmin=0.01, qmax=0.5, *, mode="chosen", device=0):
        self.n_bins = n_bins
        self.qmin = qmin
        self.qmax = qmax
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
        """BLS of every light curve over the trial periods and period
        derivatives: a list of Statistics (output='stats'), of Periodogram
        ('periodogram'), or of lists of Statistics for the top peaks
        ('peaks')."""
        validate_inputs(times, mags)
        ensure_float32(times, 'times')
        ensure_float32(mags, 'mags')
        errs = _check_errs(times, errs)
        return _calc(ALGO_BLS, (self.n_bins, self.qmin, self.qmax), self.flags, self.device,
                     times, list(mags), errs, periods, period_dts, output, True, n_stats,
                     significance_type, n_peaks, min_distance)
