# The C ABI of include/pf.h as the drop-in Cython modules call it.  Every
# call runs without the GIL; a nonzero status is raised as RuntimeError with
# pf_last_error's message.

from libc.stdint cimport int64_t, uint32_t, uint64_t


cdef extern from "pf.h" nogil:
    ctypedef struct pf_ctx:
        pass

    int PF_OK
    int PF_MODE_PLAIN
    int PF_MODE_CHOSEN

    int pf_ctx_create(pf_ctx** out, int device)
    void pf_ctx_destroy(pf_ctx* ctx)
    const char* pf_last_error(const pf_ctx* ctx)

    int pf_ce(pf_ctx* ctx, const float* const* times, const float* const* mags,
              const uint64_t* lengths, uint64_t n_curves, const float* periods,
              uint64_t n_per, const float* period_dts, uint64_t n_pdt,
              uint32_t n_phase, uint32_t n_mag, uint32_t phase_overlap,
              uint32_t mag_overlap, int mode, float* out)
    int pf_aov(pf_ctx* ctx, const float* const* times, const float* const* mags,
               const uint64_t* lengths, uint64_t n_curves, const float* periods,
               uint64_t n_per, const float* period_dts, uint64_t n_pdt,
               uint32_t n_phase, uint32_t phase_overlap, int mode, float* out)
    int pf_ls(pf_ctx* ctx, const float* const* times, const float* const* mags,
              const uint64_t* lengths, uint64_t n_curves, const float* periods,
              uint64_t n_per, const float* period_dts, uint64_t n_pdt, int mode,
              float* out)
    int pf_ce_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                    const uint64_t* lengths, uint64_t n_curves, const float* periods,
                    uint64_t n_per, const float* period_dts, uint64_t n_pdt,
                    uint32_t n_phase, uint32_t n_mag, uint32_t phase_overlap,
                    uint32_t mag_overlap, uint32_t n_peaks, uint32_t min_distance,
                    int mode, int64_t* out_idx, float* out_val)
    int pf_aov_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                     const uint64_t* lengths, uint64_t n_curves, const float* periods,
                     uint64_t n_per, const float* period_dts, uint64_t n_pdt,
                     uint32_t n_phase, uint32_t phase_overlap, uint32_t n_peaks,
                     uint32_t min_distance, int mode, int64_t* out_idx, float* out_val)
    int pf_ls_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                    const uint64_t* lengths, uint64_t n_curves, const float* periods,
                    uint64_t n_per, const float* period_dts, uint64_t n_pdt,
                    uint32_t n_peaks, uint32_t min_distance, int mode, int64_t* out_idx,
                    float* out_val)
    int pf_fpw(pf_ctx* ctx, const float* const* times, const float* const* mags,
               const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
               const float* periods, uint64_t n_per, const float* period_dts,
               uint64_t n_pdt, uint32_t n_bins, int mode, float* out)
    int pf_fpw_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                     const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
                     const float* periods, uint64_t n_per, const float* period_dts,
                     uint64_t n_pdt, uint32_t n_bins, uint32_t n_peaks,
                     uint32_t min_distance, int mode, int64_t* out_idx, float* out_val)
    int pf_bls(pf_ctx* ctx, const float* const* times, const float* const* mags,
               const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
               const float* periods, uint64_t n_per, const float* period_dts,
               uint64_t n_pdt, uint32_t n_bins, float qmin, float qmax, int mode,
               float* out)
    int pf_bls_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                     const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
                     const float* periods, uint64_t n_per, const float* period_dts,
                     uint64_t n_pdt, uint32_t n_bins, float qmin, float qmax,
                     uint32_t n_peaks, uint32_t min_distance, int mode, int64_t* out_idx,
                     float* out_val)
