// ref_shim.cu -- C entry points onto the reference's own CUDA host drivers.
//
// TEST INFRASTRUCTURE ONLY.  Linked (by oracle/Makefile, target `ref`) with
// the reference's periodfind/cuda/{ce,aov,ls,fpw,bls}.cu compiled from the reference
// checkout, it exposes exactly the calls the reference's Cython wrappers make
// (periodfind/ce.pyx:183-187, aov.pyx:166-170, ls.pyx:150-154,
// fpw.pyx:150-154), so tests can
// run the reference's CUDA path on the GPU and compare bin occupancies and
// periodograms against periodfind_b200.  The product never links this.
#include <cstdint>
#include <vector>

#include "aov.h"
#include "bls.h"
#include "ce.h"
#include "fpw.h"
#include "ls.h"

namespace {
void unpack(const float* times, const float* mags, const int64_t* offsets,
            int64_t n_curves, std::vector<float*>& t, std::vector<float*>& m,
            std::vector<size_t>& len) {
    t.resize(n_curves);
    m.resize(n_curves);
    len.resize(n_curves);
    for (int64_t c = 0; c < n_curves; c++) {
        t[c] = const_cast<float*>(times + offsets[c]);
        m[c] = const_cast<float*>(mags + offsets[c]);
        len[c] = (size_t)(offsets[c + 1] - offsets[c]);
    }
}
}  // namespace

extern "C" {

// ConditionalEntropy(n_phase, n_mag, p_overlap, m_overlap).CalcCEValsBatched
int pfref_ce(const float* times, const float* mags, const int64_t* offsets,
             int64_t n_curves, const float* periods, int64_t n_per,
             const float* pdts, int64_t n_pdt, uint32_t n_phase,
             uint32_t n_mag, uint32_t p_overlap, uint32_t m_overlap,
             float* out) {
    std::vector<float*> t, m;
    std::vector<size_t> len;
    unpack(times, mags, offsets, n_curves, t, m, len);
    ConditionalEntropy ce(n_phase, n_mag, p_overlap, m_overlap);
    ce.CalcCEValsBatched(t, m, len, periods, pdts, (size_t)n_per,
                         (size_t)n_pdt, out);
    return 0;
}

// AOV(n_bins, overlap).CalcAOVValsBatched
int pfref_aov(const float* times, const float* mags, const int64_t* offsets,
              int64_t n_curves, const float* periods, int64_t n_per,
              const float* pdts, int64_t n_pdt, uint32_t n_bins,
              uint32_t overlap, float* out) {
    std::vector<float*> t, m;
    std::vector<size_t> len;
    unpack(times, mags, offsets, n_curves, t, m, len);
    AOV aov(n_bins, overlap);
    aov.CalcAOVValsBatched(t, m, len, periods, pdts, (size_t)n_per,
                           (size_t)n_pdt, out);
    return 0;
}

// LombScargle().CalcLSBatched
int pfref_ls(const float* times, const float* mags, const int64_t* offsets,
             int64_t n_curves, const float* periods, int64_t n_per,
             const float* pdts, int64_t n_pdt, float* out) {
    std::vector<float*> t, m;
    std::vector<size_t> len;
    unpack(times, mags, offsets, n_curves, t, m, len);
    LombScargle ls;
    ls.CalcLSBatched(t, m, len, periods, pdts, (size_t)n_per, (size_t)n_pdt,
                     out);
    return 0;
}

// FPW(n_bins).CalcFPWBatched; errs is packed like mags (unit errors are
// passed explicitly, as the Cython wrapper does for errs=None).
int pfref_fpw(const float* times, const float* mags, const float* errs,
              const int64_t* offsets, int64_t n_curves, const float* periods,
              int64_t n_per, const float* pdts, int64_t n_pdt, uint32_t n_bins,
              float* out) {
    std::vector<float*> t, m, e;
    std::vector<size_t> len;
    unpack(times, mags, offsets, n_curves, t, m, len);
    e.resize(n_curves);
    for (int64_t c = 0; c < n_curves; c++) e[c] = const_cast<float*>(errs + offsets[c]);
    FPW fpw(n_bins);
    fpw.CalcFPWBatched(t, m, e, len, periods, pdts, (size_t)n_per, (size_t)n_pdt, out);
    return 0;
}

// BLS(n_bins, qmin, qmax).CalcBLSBatched; errs packed like mags.
int pfref_bls(const float* times, const float* mags, const float* errs,
              const int64_t* offsets, int64_t n_curves, const float* periods,
              int64_t n_per, const float* pdts, int64_t n_pdt, uint32_t n_bins, float qmin,
              float qmax, float* out) {
    std::vector<float*> t, m, e;
    std::vector<size_t> len;
    unpack(times, mags, offsets, n_curves, t, m, len);
    e.resize(n_curves);
    for (int64_t c = 0; c < n_curves; c++) e[c] = const_cast<float*>(errs + offsets[c]);
    BLS bls(n_bins, qmin, qmax);
    bls.CalcBLSBatched(t, m, e, len, periods, pdts, (size_t)n_per, (size_t)n_pdt, out);
    return 0;
}

// The reference's CE histogram step alone (ce.cu:262-290, one curve,
// device pointers): normalised histograms, count / (N * po * mo), as f32.
int pfref_ce_hists(const float* d_times, const float* d_mags, uint64_t length,
                   const float* d_periods, const float* d_pdts, uint64_t n_per,
                   uint64_t n_pdt, uint32_t n_phase, uint32_t n_mag,
                   uint32_t p_overlap, uint32_t m_overlap, float* h_out) {
    ConditionalEntropy ce(n_phase, n_mag, p_overlap, m_overlap);
    float* d = ce.DeviceFoldAndBin(d_times, d_mags, (size_t)length, d_periods,
                                   d_pdts, (size_t)n_per, (size_t)n_pdt);
    size_t bytes = (size_t)n_phase * n_mag * n_per * n_pdt * sizeof(float);
    cudaError_t e = cudaMemcpy(h_out, d, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : -1;
}

// The reference's AOV bin step alone (aov.cu:265-299, one curve, device
// pointers): per-bin (count, sum, sq_sum) written as 3 x u32/f32 words.
int pfref_aov_bins(const float* d_times, const float* d_mags, uint64_t length,
                   const float* d_periods, const float* d_pdts, uint64_t n_per,
                   uint64_t n_pdt, uint32_t n_bins, uint32_t overlap,
                   void* h_out) {
    AOV aov(n_bins, overlap);
    AOVData* d = aov.DeviceFoldAndBin(d_times, d_mags, (size_t)length,
                                      d_periods, d_pdts, (size_t)n_per,
                                      (size_t)n_pdt);
    size_t bytes = (size_t)n_bins * n_per * n_pdt * sizeof(AOVData);
    cudaError_t e = cudaMemcpy(h_out, d, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : -1;
}

}  // extern "C"
