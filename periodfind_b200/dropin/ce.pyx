#cython: language_level=3
"""Conditional Entropy on the B200, in place of periodfind's ce.pyx.

Same class, constructor and calc() as periodfind/ce.pyx:41-209; the
periodograms come from the C ABI of include/pf.h (pf_ce, pf_ce_peaks)
instead of the reference's CalcCEValsBatched (ce.pyx:25-39).  Additions:
output='peaks' (with n_peaks, min_distance, as the CPU classes have it) and
the keyword-only constructor arguments mode ('chosen', default, or
'plain': the reference's fold operation for operation) and device.
"""

include "_common.pxi"


cdef class ConditionalEntropy:
    """Conditional Entropy periodogram of folded (phase, magnitude)
    histograms, n_phase x n_mag bins; each entry widened over
    phase_bin_extent x mag_bin_extent neighbouring bins with wrap-around.
    The minimum is the best period."""

    cdef readonly int n_phase, n_mag, phase_bin_extent, mag_bin_extent, device
    cdef readonly str mode
    cdef int flags

    def __cinit__(self, n_phase=10, n_mag=10, phase_bin_extent=1, mag_bin_extent=1, *,
                  mode="chosen", device=0):
        self.n_phase = n_phase
        self.n_mag = n_mag
        self.phase_bin_extent = phase_bin_extent
        self.mag_bin_extent = mag_bin_extent
        self.mode = mode
        self.flags = _mode_flags(mode)
        self.device = device

    def calc(self,
             list times,
             list mags,
             cnp.ndarray[ndim=1, dtype=cnp.float32_t] periods,
             cnp.ndarray[ndim=1, dtype=cnp.float32_t] period_dts,
             output="stats",
             normalize=True,
             center=False,
             n_stats=1,
             significance_type='stdmean',
             n_peaks=N_PEAKS_DEFAULT,
             min_distance=MIN_DISTANCE_DEFAULT):
        """Conditional Entropy of every light curve over the trial periods
        and period derivatives: a list of Statistics (output='stats'), of
        Periodogram ('periodogram'), or of lists of Statistics for the top
        peaks ('peaks').  Magnitudes are normalised into (0, 1) by default,
        as the histogram needs."""
        validate_inputs(times, mags)
        ensure_float32(times, 'times')
        ensure_float32(mags, 'mags')
        mags_use = prepare_magnitudes(mags, center, normalize)
        return _calc(ALGO_CE, (self.n_phase, self.n_mag, self.phase_bin_extent,
                               self.mag_bin_extent), self.flags, self.device, times,
                     list(mags_use), None, periods, period_dts, output, False, n_stats,
                     significance_type, n_peaks, min_distance)
