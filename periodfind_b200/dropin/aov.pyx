#cython: language_level=3
"""Analysis of Variance on the B200, in place of periodfind's aov.pyx.

Same class, constructor and calc() as periodfind/aov.pyx:38-192; the
periodograms come from the C ABI of include/pf.h (pf_aov, pf_aov_peaks)
instead of the reference's CalcAOVValsBatched (aov.pyx:24-36).  Additions:
output='peaks' (n_peaks, min_distance) and the keyword-only constructor
arguments mode ('chosen' or 'plain') and device.
"""

include "_common.pxi"


cdef class AOV:
    """Analysis-of-Variance periodogram over n_phase phase bins, each entry
    widened over phase_bin_extent bins with wrap-around.  The maximum is the
    best period."""

    cdef readonly int n_phase, phase_bin_extent, device
    cdef readonly str mode
    cdef int flags

    def __cinit__(self, n_phase=10, phase_bin_extent=1, *, mode="chosen", device=0):
        self.n_phase = n_phase
        self.phase_bin_extent = phase_bin_extent
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
             center=False,
             n_stats=1,
             significance_type='stdmean',
             n_peaks=N_PEAKS_DEFAULT,
             min_distance=MIN_DISTANCE_DEFAULT):
        """AOV of every light curve over the trial periods and period
        derivatives: a list of Statistics (output='stats'), of Periodogram
        ('periodogram'), or of lists of Statistics for the top peaks
        ('peaks')."""
        validate_inputs(times, mags)
        ensure_float32(times, 'times')
        ensure_float32(mags, 'mags')
        mags_use = prepare_magnitudes(mags, center, normalize)
        return _calc(ALGO_AOV, (self.n_phase, self.phase_bin_extent), self.flags, self.device,
                     times, list(mags_use), None, periods, period_dts, output, True, n_stats,
                     significance_type, n_peaks, min_distance)
