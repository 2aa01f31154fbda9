// pf_launch.h -- host-side entry points into the kernel translation units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "pf_types.h"

namespace pfk {

// KIND_LSREC: Lomb-Scargle on a uniform frequency grid with the
// angle-addition recurrence along the grid (pf_lsrec.cuh); `rounds` holds
// its frequencies per thread.
// KIND_BINWARP: the chosen CE / AOV binning with one shared histogram per
// warp and trial period, filled with shared atomics (pf_binwarp.cuh), the
// alternative to KIND_BIN's per-thread privatised histograms.
enum : int { KIND_FOLD = 0, KIND_BIN = 1, KIND_LSREC = 2, KIND_BINWARP = 3 };
constexpr uint32_t kWarpMaxPoints = 1024;  // KIND_BINWARP: longest curve it stages
constexpr uint32_t kRecTileBytes = 512 * 16;  // lsrec_kernel's staged points

// Kernels that take their items from the device work queue (a curve order;
// the device derives the items): the chosen bin kernel and the chosen folds.
// Each runs either persistently (a fixed grid pulling items from an atomic
// counter) or statically (one CTA per item).  The reference fold and the
// all-FP32 study fold take one CTA per item of a host-built list.
__host__ __device__ constexpr bool uses_queue(int kind, int fold) {
    return kind == KIND_BIN || kind == KIND_LSREC || kind == KIND_BINWARP || fold == FOLD_EXACT ||
           fold == FOLD_DF;
}

struct FoldConfig {
    int kind;   // KIND_FOLD: fold_kernel; KIND_BIN: the chosen CE/AOV bin_kernel
    bool cnt16; // bin_kernel CE: 16-bit counters
    int algo;   // ALGO_*
    int fold;   // FOLD_*
    int acc;    // AOVACC_* (AOV only)
    int block;  // threads per CTA: 64, 128 or 256
    bool ovl;   // general bin-overlap path
    bool ref_stats; // bin_kernel: the reference's statistic operation sequence
    bool persist;   // queue kernels: persistent grid instead of one CTA per item
    int rounds;     // bin kernel: an item is rounds x block periods (1 or 4);
                    // KIND_LSREC: frequencies per thread (4 or 8)
    int n_sm;       // persistent kernels: grid = n_sm x resident CTAs per SM
};

size_t fold_smem(const FoldConfig& c, uint32_t n_phase, uint32_t n_mag);

// Periods in one work item of a queue kernel.
inline int item_periods(const FoldConfig& c) {
    return c.block * ((c.kind == KIND_BIN || c.kind == KIND_LSREC) && c.rounds > 1 ? c.rounds : 1);
}

// Semantics of the reference's CUDA build (-use_fast_math).
cudaError_t launch_fold_cudasem(const FoldConfig& c, const FoldParams& p, uint32_t n_work,
                                cudaStream_t stream);
cudaError_t launch_magbin_cudasem(const float* m, uint32_t* aux, const CurveDesc* curves,
                                  uint32_t n_curves, uint32_t n_mag, float mag_bin_size,
                                  int flag_saturated, cudaStream_t stream);
// Semantics of the reference's CPU path (IEEE, no contraction).
cudaError_t launch_fold_cpusem(const FoldConfig& c, const FoldParams& p, uint32_t n_work,
                               cudaStream_t stream);
cudaError_t launch_magbin_cpusem(const float* m, uint32_t* aux, const CurveDesc* curves,
                                 uint32_t n_curves, uint32_t n_mag, float mag_bin_size,
                                 int flag_saturated, cudaStream_t stream);

cudaError_t launch_binaux_cudasem(const float* m, void* aux, const CurveDesc* curves,
                                  uint32_t n_curves, uint32_t n_mag, float mag_bin_size,
                                  int block, int cnt16, cudaStream_t s);
cudaError_t launch_binaux_cpusem(const float* m, void* aux, const CurveDesc* curves,
                                 uint32_t n_curves, uint32_t n_mag, float mag_bin_size,
                                 int block, int cnt16, cudaStream_t s);

// FPW and BLS (pf_fpw.cuh): per point t, inverse variance iv = 1 / err^2 and
// ivy = iv * m, packed per curve at off[c] with len[c] points; out is
// [curve][period][pdt].  bin_size = 1 / n_bins as the reference rounds it.
struct FpwParams {
    const float* t;
    const float* iv;
    const float* ivy;
    const int64_t* off;
    const uint32_t* len;
    const float* periods;
    const float* pdts;
    uint64_t n_per;
    uint32_t n_pdt;
    uint32_t n_bins;
    float bin_size;
    float* out;
    double tmax;      // max |t| over the batch (the chosen form's range guard)
    uint32_t edge_d;  // bin-edge guard, units of 2^-20 bin (as the CE / AOV bin kernels)
    int bls;          // BLS instead of FPW (ivy then holds w * (m - weighted mean))
    uint32_t nb_min, nb_max;  // BLS: window widths searched, in bins
};
constexpr uint32_t kFpwMaxBins = 128;
// exact: the chosen form (fast bins with the reference sequence near bin
// edges; the same values).
cudaError_t launch_fpw_cudasem(const FpwParams& p, bool exact, uint64_t n_curves,
                               cudaStream_t s);
cudaError_t launch_fpw_cpusem(const FpwParams& p, bool exact, uint64_t n_curves,
                              cudaStream_t s);

// Folded phase of every (period, time) pair with one fold variant
// (FOLD_REF / FOLD_EXACT / FOLD_F32 / FOLD_DF), out[p * n + i].
cudaError_t launch_phase_probe_cudasem(int fold, const float* t, uint64_t n,
                                       const float* periods, uint64_t n_per, float period_dt,
                                       float* out, cudaStream_t s);
cudaError_t launch_phase_probe_cpusem(int fold, const float* t, uint64_t n,
                                      const float* periods, uint64_t n_per, float period_dt,
                                      float* out, cudaStream_t s);

// Preparation kernels (pf_prep.cu).
// max |t| over n packed points into *tmax_bits (float bits; zeroed first).
cudaError_t launch_tmax(const float* t, size_t n, unsigned* tmax_bits, cudaStream_t stream);
// AOV bin kernel: 32-bit fixed-point magnitudes (k bits) and per-curve sums.
cudaError_t launch_aov_fix32_prep(const float* m, uint32_t* aux32, CurveDesc* curves,
                                  uint32_t n_curves, cudaStream_t stream);
cudaError_t launch_aov_mean(const float* m, CurveDesc* curves, uint32_t n_curves,
                            cudaStream_t stream);
cudaError_t launch_aov_fix_prep(const float* m, uint64_t* aux64, CurveDesc* curves,
                                uint32_t n_curves, uint32_t overlap, cudaStream_t stream);

cudaError_t launch_pack(const float* src_t, const float* src_m, const int64_t* src_off,
                        const CurveDesc* curves, uint32_t n_curves, float* dst_t, float* dst_m,
                        cudaStream_t stream);

// Lomb-Scargle derivatives (pf_lsgrad.cu).  Times and magnitudes are CSR
// arrays with device offsets; omega is angular frequency (rad / time unit),
// omega[c * omega_stride + k] (stride 0: one grid for every curve).
// Outputs are [n_curves][n_freq]; coef holds (alpha, beta) pairs.
struct LsEvalParams {
    const float* t = nullptr;
    const float* y = nullptr;
    const int64_t* off = nullptr;
    uint64_t n_curves = 0;
    const double* omega = nullptr;
    uint64_t omega_stride = 0;
    uint64_t n_freq = 0;
    float* power = nullptr;
    float* dpdw = nullptr;
    float* d2pdw2 = nullptr;
    float* coef = nullptr;
    // Newton refinement only
    const double* half_width = nullptr;  // [n_curves][n_freq] bracket half-width
    uint32_t n_steps = 0;
    double* omega_out = nullptr;
};
struct LsGradParams {
    const float* t = nullptr;
    const int64_t* off = nullptr;
    uint64_t n_curves = 0;
    const double* omega = nullptr;
    uint64_t omega_stride = 0;
    uint64_t n_freq = 0;
    const float* grad_power = nullptr;
    const float* dpdw = nullptr;
    const float* coef = nullptr;
    double* grad_omega = nullptr;
    float* grad_mags = nullptr;
};
cudaError_t launch_ls_eval(const LsEvalParams& p, int order, cudaStream_t stream);
cudaError_t launch_ls_refine(const LsEvalParams& p, cudaStream_t stream);
cudaError_t launch_ls_grad(const LsGradParams& p, uint32_t max_len, cudaStream_t stream);

// 'stats' output (pf_stats.cu): per row of [n_curves][n_cells], numpy's
// mean / std / median / MAD into stats[4 * c + {0..3}] and the n_top best
// cells, best first (use_max: largest).  stats_leaf_count is the number of
// leaves of numpy's pairwise summation over n elements (12 B of shared
// memory each).
uint32_t stats_leaf_count(uint32_t n);
// Magnitude preparation on the device (kind 1: centre, 2: normalise) as
// numpy does it; curve c is m[d_off[c] .. d_off[c+1]); leaf_cap is the
// largest stats_leaf_count over the curves (kind 1).
cudaError_t launch_prep_mags(const float* m, const int64_t* d_off, uint64_t n_curves,
                             uint32_t leaf_cap, int kind, float* out, cudaStream_t s);
cudaError_t launch_stats(const float* pg, uint64_t n_curves, uint32_t n_cells, int use_max,
                         uint32_t n_top, float* stats, int64_t* top_idx, float* top_val,
                         cudaStream_t stream);

// Peak search (pf_peaks.cu): one CTA per curve over a [n_curves][flat]
// periodogram; rust/src/peaks.rs semantics.
cudaError_t launch_peaks(const float* pg, uint64_t n_curves, uint64_t flat_len,
                         uint32_t n_peaks, uint32_t min_distance, int use_max,
                         int64_t* out_idx, float* out_val, cudaStream_t stream);

}  // namespace pfk
