#cython: language_level=3
"""Lomb-Scargle on the B200, in place of periodfind's ls.pyx.

Same class, constructor and calc() as periodfind/ls.pyx:37-176; the
periodograms come from the C ABI of include/pf.h (pf_ls, pf_ls_peaks)
instead of the reference's CalcLSBatched (ls.pyx:24-35).  Additions:
output='peaks' (n_peaks, min_distance) and the keyword-only constructor
arguments mode ('chosen': split-precision phase; 'plain': the reference's
FP64-divide fold) and device.
"""

include "_common.pxi"


cdef class LombScargle:
    """Lomb-Scargle periodogram; magnitudes centred by default.  The
    maximum is the best period."""

    cdef readonly int device
    cdef readonly str mode
    cdef int flags

    def __cinit__(self, *, mode="chosen", device=0):
        self.mode = mode
        self.flags = _mode_flags(mode)
        self.device = device

    def calc(self,
             list times,
             list mags,
             cnp.ndarray[ndim=1, dtype=cnp.float32_t] periods,
             cnp.ndarray[ndim=1, dtype=cnp.float32_t] period_dts,
             output="stats",
             normalize=False,
             center=True,
             n_stats=1,
             significance_type='stdmean',
             n_peaks=N_PEAKS_DEFAULT,
             min_distance=MIN_DISTANCE_DEFAULT):
        """Lomb-Scargle power of every light curve over the trial periods
        and period derivatives: a list of Statistics (output='stats'), of
        Periodogram ('periodogram'), or of lists of Statistics for the top
        peaks ('peaks')."""
        validate_inputs(times, mags)
        ensure_float32(times, 'times')
        ensure_float32(mags, 'mags')
        mags_use = prepare_magnitudes(mags, center, normalize)
        return _calc(ALGO_LS, (), self.flags, self.device, times, list(mags_use), None,
                     periods, period_dts, output, True, n_stats, significance_type, n_peaks,
                     min_distance)
