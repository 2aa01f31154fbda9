/*
 * pf.h -- C ABI of periodfind_b200, a B200 (sm_100a) implementation of
 * periodfind's batched periodogram hot path: Conditional Entropy (CE),
 * Analysis of Variance (AOV) and Lomb-Scargle (LS) over every
 * (light curve x trial period x period derivative).
 *
 * Conventions
 *  - Every function returns PF_OK (0) or a negative PF_E* code and never
 *    exits the process; pf_last_error() describes the last failure.
 *  - Host-pointer entry points take the same arguments the reference's
 *    Cython wrappers pass to its C++ drivers: one host array per curve for
 *    times and magnitudes, the curve lengths, the trial periods and period
 *    derivatives, and a caller-owned output of n_curves * n_per * n_pdt
 *    floats laid out [curve][period][pdt] (C order).  Magnitudes are used as
 *    given: centring / normalisation is the caller's job, as in the
 *    reference (periodfind/ce.pyx:167).
 *  - A context owns its device buffers, pinned staging, stream and tuning
 *    cache.  A context is used by one host thread at a time; distinct
 *    contexts may run concurrently.
 *  - Times must be finite (checked, PF_EINVAL).  Empty curves are allowed
 *    and produce the reference CPU path's values (CE NaN, AOV 0, LS 0).
 *
 * mode bits
 *  PF_MODE_PLAIN   the reference's fold operation for operation: an FP64
 *                  divide per (point, period) (periodfind/cuda/ce.cu:141-143).
 *  PF_MODE_CHOSEN  the tuned form.  CE/AOV: the reference's quotient without
 *                  a divide (bit-identical), bins from FP64/integer ops with
 *                  the reference's exact sequence near bin edges (identical
 *                  bin occupancies), 16-bit CE counters, exact fixed-point
 *                  AOV sums.  LS: split-precision FP32 phase, no FP64 per
 *                  point, with the error bound of the reference's FP64 fold
 *                  (the f32 rounding of the phase, <= 2^-25 turns).
 *  PF_SEM_CPU      arithmetic of the reference's CPU (Rust) path: IEEE
 *                  divides, no multiply-add contraction, accurate libm-style
 *                  log/sin/cos.  Without it the arithmetic follows the
 *                  reference's CUDA build (compiled with -use_fast_math).
 *  PF_FOLD_F32     (LS precision study) fold t/P entirely in FP32.
 *  PF_FOLD_DF      (LS) split-precision FP32 phase frac(t * f) with the
 *                  frequency as an unevaluated float pair; no FP64 per point.
 *  PF_FOLD_EXACT   (LS, chosen) the divide-free exact fold instead of the
 *                  split-precision phase: bit-identical to the plain form.
 *  PF_TIMING       record device timestamps per work item (CTA start and
 *                  end, %globaltimer) for pf_curve_latency.
 *  PF_NO_TUNE      (chosen) skip the launch-shape autotuner and use the
 *                  default shape for every length class.  The chosen kernels
 *                  take their work from a device queue split by curve length
 *                  ([0,64), [64,256), [256,1024), [1024,4096), [4096,...));
 *                  the first call that meets a (computation, class) pair
 *                  times the candidate shapes on a sample of that class and
 *                  synchronises the stream once; the result is cached in the
 *                  context.  Results do not depend on the shape.
 *  PF_REF_STATS    (CE/AOV, chosen) compute the statistic from the bins with
 *                  the reference's operation sequence instead of the chosen
 *                  form's divide-free one (agreeing to ~1e-6): values are then
 *                  bit-identical to the plain form exactly when the bin
 *                  occupancies are, which is how occupancy parity is tested.
 *  PF_ASYNC        (pf_ce_peaks / pf_aov_peaks / pf_ls_peaks / pf_fpw_peaks /
 *                  pf_bls_peaks only) enqueue
 *                  and return: the inputs are packed into the context's
 *                  staging block and the work is queued on the context's
 *                  stream, but out_idx / out_val are written later, by the
 *                  pf_wait call that collects this call.  The caller keeps
 *                  them alive until then.  At most two PF_ASYNC calls may be
 *                  pending on a context; a third is PF_EINVAL.  A caller
 *                  packs the next batch while the GPU runs this one.  Not
 *                  with PF_TIMING.
 *  PF_TRIG_SINCOS / PF_TRIG_RECURRENCE  (pf_ls_fgrid*, chosen) keep one trig
 *                  form instead of letting the autotuner pick per length
 *                  class: MUFU sine / cosine at every (point, frequency), or
 *                  one sine / cosine per point and thread followed by
 *                  angle-addition rotations along the uniform grid.
 *  PF_BINS_SHARED  (CE / AOV, chosen) keep the shared-histogram binning
 *                  (one histogram per warp and trial period, filled with
 *                  shared atomics) for the length classes it serves (curves
 *                  shorter than 1024 points) instead of letting the
 *                  autotuner weigh it against per-thread privatised
 *                  histograms.  Values are identical either way.
 *  PF_ONE_LAUNCH   (chosen) run every curve in one launch with the shape
 *                  tuned for the length class holding the most points,
 *                  instead of one launch per class with its own tuned shape
 *                  (for comparison; values are identical).
 *  PF_HOST_NORMALIZE / PF_HOST_CENTER  (host-pointer periodogram, peak and
 *                  stats calls) prepare the magnitudes while packing them,
 *                  as pf_normalize_mags / pf_center_mags would (numpy's
 *                  values): the caller passes raw magnitudes and saves a
 *                  pass and a copy.  Empty curves are left as they are.
 */
#ifndef PERIODFIND_B200_PF_H
#define PERIODFIND_B200_PF_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PF_OK 0
#define PF_EINVAL (-1)       /* bad argument                              */
#define PF_ECUDA (-2)        /* CUDA runtime error                        */
#define PF_ENOMEM (-3)       /* device or pinned allocation failed        */
#define PF_EUNSUPPORTED (-4) /* valid but unsupported configuration       */
#define PF_ETIMEOUT (-5)     /* a bounded device wait gave up             */

#define PF_MODE_PLAIN 0x0
#define PF_MODE_CHOSEN 0x1
#define PF_SEM_CPU 0x10
#define PF_FOLD_F32 0x100
#define PF_FOLD_DF 0x200
#define PF_FOLD_EXACT 0x400
#define PF_TIMING 0x1000
#define PF_REF_STATS 0x2000
#define PF_NO_TUNE 0x4000
#define PF_ASYNC 0x8000
#define PF_TRIG_SINCOS 0x10000
#define PF_TRIG_RECURRENCE 0x20000
#define PF_BINS_SHARED 0x40000
#define PF_ONE_LAUNCH 0x80000
#define PF_HOST_NORMALIZE 0x100000
#define PF_HOST_CENTER 0x200000

typedef struct pf_ctx pf_ctx;

/* Library version, major * 10000 + minor * 100 + patch. */
int pf_version(void);

/* Create a context on CUDA device `device`. */
int pf_ctx_create(pf_ctx** out, int device);
void pf_ctx_destroy(pf_ctx* ctx);
/* Message for the last failure on this context ("" if none).  With a NULL
 * context, the message of the last failed pf_ctx_create on this thread. */
const char* pf_last_error(const pf_ctx* ctx);

/* ---------------------------------------------------------- periodograms */

/* Replaces ConditionalEntropy::CalcCEValsBatched
 * (periodfind/cuda/ce.h, ce.cu:420-562; bound at periodfind/ce.pyx:25-39).
 * n_phase x n_mag histogram with phase_overlap / mag_overlap bin extents.
 * Magnitudes are bin coordinates meant to lie in [0, 1) (normalise first).
 * Values outside are accepted, as the reference accepts them (its own tests
 * centre CE magnitudes, tests/test_periodfind.py:535-546): a negative value
 * falls in magnitude bin 0 (the float-to-integer conversion saturates, as
 * in the reference's CUDA and Rust paths) and a value >= 1 wraps modulo
 * n_mag.  That is memory-safe, where the reference writes outside the
 * curve's bins (periodfind/cuda/ce.cu:66-77).  Minimum is best. */
int pf_ce(pf_ctx* ctx, const float* const* times, const float* const* mags,
          const uint64_t* lengths, uint64_t n_curves, const float* periods,
          uint64_t n_per, const float* period_dts, uint64_t n_pdt,
          uint32_t n_phase, uint32_t n_mag, uint32_t phase_overlap,
          uint32_t mag_overlap, int mode, float* out);

/* Replaces AOV::CalcAOVValsBatched (periodfind/cuda/aov.h, aov.cu:429-576;
 * bound at periodfind/aov.pyx:24-36).  Maximum is best. */
int pf_aov(pf_ctx* ctx, const float* const* times, const float* const* mags,
           const uint64_t* lengths, uint64_t n_curves, const float* periods,
           uint64_t n_per, const float* period_dts, uint64_t n_pdt,
           uint32_t n_phase, uint32_t phase_overlap, int mode, float* out);

/* Replaces LombScargle::CalcLSBatched (periodfind/cuda/ls.h, ls.cu:232-359;
 * bound at periodfind/ls.pyx:24-35).  Maximum is best. */
int pf_ls(pf_ctx* ctx, const float* const* times, const float* const* mags,
          const uint64_t* lengths, uint64_t n_curves, const float* periods,
          uint64_t n_per, const float* period_dts, uint64_t n_pdt, int mode,
          float* out);

/* Lomb-Scargle on a uniform frequency grid (no counterpart in the
 * reference, whose grid is an array of trial periods): trial frequency k is
 * f_min + k * df exactly, k < n_freq (cycles per time unit), one period
 * derivative (0); out is [curve][k].  On such a grid the phases of one point
 * advance by the same angle from one frequency to the next, so besides the
 * MUFU sine / cosine per evaluation the autotuner can pick, per length
 * class, an angle-addition recurrence along the grid (PF_TRIG_* forces one).
 * Chosen form only (PF_MODE_CHOSEN; PF_FOLD_EXACT for an FP64 phase);
 * CUDA arithmetic only (PF_SEM_CPU is PF_EUNSUPPORTED).  Magnitudes as
 * pf_ls.  The device-pointer variant takes CSR curves as pf_ls_dev. */
int pf_ls_fgrid(pf_ctx* ctx, const float* const* times, const float* const* mags,
                const uint64_t* lengths, uint64_t n_curves, double f_min, double df,
                uint64_t n_freq, int mode, float* out);
int pf_ls_fgrid_dev(pf_ctx* ctx, const float* d_times, const float* d_mags,
                    const int64_t* offsets, uint64_t n_curves, double f_min, double df,
                    uint64_t n_freq, int mode, float* d_out, void* stream);

/* The bins behind a CE or AOV periodogram, for occupancy checks: the
 * counterpart of ConditionalEntropy::FoldAndBin (periodfind/cuda/ce.h:194,
 * ce.cu:262-290, which returns count / (N * po * mo) per bin) and
 * AOV::FoldAndBin (periodfind/cuda/aov.h:132, whose AOVData holds the
 * count per bin).  algo is PF_ALGO_CE or PF_ALGO_AOV (n_mag and
 * mag_overlap are ignored for AOV).  Computes the periodogram into `out`
 * as pf_ce / pf_aov do and writes the raw u32 count of every bin of every
 * cell into out_counts, [curve][period][pdt][bin] with bin = phase_bin *
 * n_mag + mag_bin (CE) or phase_bin (AOV): n_curves * n_per * n_pdt *
 * (n_phase * n_mag or n_phase) entries.  With PF_MODE_CHOSEN the counts come
 * from the chosen kernels with PF_REF_STATS implied.  PF_ASYNC and
 * PF_TIMING are rejected. */
int pf_bin_counts(pf_ctx* ctx, int algo, const float* const* times,
                  const float* const* mags, const uint64_t* lengths, uint64_t n_curves,
                  const float* periods, uint64_t n_per, const float* period_dts,
                  uint64_t n_pdt, uint32_t n_phase, uint32_t n_mag, uint32_t phase_overlap,
                  uint32_t mag_overlap, int mode, float* out, uint32_t* out_counts);

/* ----------------------------------------------------------------- peaks */

/* Periodogram + top-N peak search without returning the periodogram.
 * Replaces calc_{ce,aov,ls}_peaks_batched (rust/src/lib.rs:559-677, used by
 * periodfind/cpu/__init__.py:148-161, :255-266, :352-362) with the peak
 * semantics of rust/src/peaks.rs:18-238 on the flattened [period][pdt]
 * grid: strict interior local extrema (minima for CE, maxima for AOV/LS),
 * greedy min_distance, sorted best-first.  out_idx / out_val are
 * [n_curves][n_peaks]; unused slots hold index -1 and value 0. */
int pf_ce_peaks(pf_ctx* ctx, const float* const* times,
                const float* const* mags, const uint64_t* lengths,
                uint64_t n_curves, const float* periods, uint64_t n_per,
                const float* period_dts, uint64_t n_pdt, uint32_t n_phase,
                uint32_t n_mag, uint32_t phase_overlap, uint32_t mag_overlap,
                uint32_t n_peaks, uint32_t min_distance, int mode,
                int64_t* out_idx, float* out_val);
int pf_aov_peaks(pf_ctx* ctx, const float* const* times,
                 const float* const* mags, const uint64_t* lengths,
                 uint64_t n_curves, const float* periods, uint64_t n_per,
                 const float* period_dts, uint64_t n_pdt, uint32_t n_phase,
                 uint32_t phase_overlap, uint32_t n_peaks,
                 uint32_t min_distance, int mode, int64_t* out_idx,
                 float* out_val);
int pf_ls_peaks(pf_ctx* ctx, const float* const* times,
                const float* const* mags, const uint64_t* lengths,
                uint64_t n_curves, const float* periods, uint64_t n_per,
                const float* period_dts, uint64_t n_pdt, uint32_t n_peaks,
                uint32_t min_distance, int mode, int64_t* out_idx,
                float* out_val);

/* FPW, the fast phase-folding weighted statistic (Finkbeiner et al. 2025).
 * Replaces FPW::CalcFPWBatched (periodfind/cuda/fpw.h, fpw.cu; bound at
 * periodfind/fpw.pyx:14-26) and calc_fpw_batched / calc_fpw_peaks_batched
 * (rust/src/lib.rs:202-256, 680-720).  Per point w = 1 / err^2 (errs NULL,
 * or errs[c] NULL: err = 1); per phase bin V = sum w, Y = sum w * m; value
 * sum over bins with V > 0 of Y^2 / (2 V).  Maximum is best.  n_bins in
 * [1, 128].  Magnitudes are used as given.  PF_MODE_CHOSEN folds without a
 * divide (same values); PF_SEM_CPU takes the Rust path's bin rule and IEEE
 * arithmetic.  PF_TIMING is refused; PF_ASYNC applies to pf_fpw_peaks. */
int pf_fpw(pf_ctx* ctx, const float* const* times, const float* const* mags,
           const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
           const float* periods, uint64_t n_per, const float* period_dts, uint64_t n_pdt,
           uint32_t n_bins, int mode, float* out);
int pf_fpw_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                 const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
                 const float* periods, uint64_t n_per, const float* period_dts, uint64_t n_pdt,
                 uint32_t n_bins, uint32_t n_peaks, uint32_t min_distance, int mode,
                 int64_t* out_idx, float* out_val);

/* BLS, box least squares (Kovacs, Zucker & Mazeh 2002).  Replaces
 * BLS::CalcBLSBatched (periodfind/cuda/bls.h, bls.cu; bound at
 * periodfind/bls.pyx:20-33) and calc_bls_batched / calc_bls_peaks_batched
 * (rust/src/lib.rs:264-322, 718-760).  Per point w = 1 / err^2 (errs NULL:
 * err = 1) and w * (m - mean), mean = sum(w m) / sum(w) in sequential f32
 * sums; per phase bin W and Y; the value is the best s^2 / (r (W_total - r))
 * over windows of nb_min .. nb_max consecutive bins (wrapping; nb_min =
 * max(floor(qmin n_bins), 1), nb_max = min(ceil(qmax n_bins), n_bins - 1))
 * whose weight fraction r / W_total lies in (0, 1).  Maximum is best.
 * n_bins in [1, 128]; modes as pf_fpw (PF_ASYNC: pf_bls_peaks). */
int pf_bls(pf_ctx* ctx, const float* const* times, const float* const* mags,
           const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
           const float* periods, uint64_t n_per, const float* period_dts, uint64_t n_pdt,
           uint32_t n_bins, float qmin, float qmax, int mode, float* out);
int pf_bls_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                 const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
                 const float* periods, uint64_t n_per, const float* period_dts, uint64_t n_pdt,
                 uint32_t n_bins, float qmin, float qmax, uint32_t n_peaks,
                 uint32_t min_distance, int mode, int64_t* out_idx, float* out_val);

/* Magnitude preparation on the device for device-resident curves (curve c
 * is d_mags[offsets[c] .. offsets[c+1]), offsets on the host), with the
 * values the reference's prepare_magnitudes gets from numpy on the host
 * (periodfind/_utils.py:29-45), bit for bit: PF_PREP_CENTER writes
 * m - np.mean(m) (numpy's pairwise float32 sum), PF_PREP_NORMALIZE writes
 * ((m - min) / (max - min)) * 0.999 + 5e-4 in float32 (NaN propagating).
 * d_out may equal d_mags.  Enqueued on `stream` (NULL: the default stream);
 * a later call on this context waits for this one's kernel before it
 * rewrites the context's copy of the offsets.  No reference counterpart:
 * the reference prepares magnitudes with numpy on the host. */
#define PF_PREP_CENTER 1
#define PF_PREP_NORMALIZE 2
int pf_prepare_mags_dev(pf_ctx* ctx, const float* d_mags, const int64_t* offsets,
                        uint64_t n_curves, int kind, float* d_out, void* stream);

/* Collect the oldest pending PF_ASYNC peak call on this context: wait for
 * its work, then write its peaks into the out_idx / out_val it was given.
 * Calls are collected in the order they were made.  PF_EINVAL when none is
 * pending; a device error of the collected call is returned here.  No
 * reference counterpart (the reference's calls are synchronous). */
int pf_wait(pf_ctx* ctx);

/* Periodogram + the 'stats' output computed on the device: what the
 * reference's Statistics.statistics_from_data (periodfind/__init__.py:
 * 338-400) derives from each curve's periodogram with numpy, with numpy's
 * results bit for bit -- out_stats[4 * c + {0, 1, 2, 3}] = np.mean, np.std
 * (float32, numpy's pairwise summation order), np.median, and the median of
 * |data - median|; out_idx / out_val [n_curves][n_top] = the n_top best cells
 * of the flattened [period][pdt] grid (smallest for CE, largest for AOV / LS;
 * NaN ranks largest), best first, ties by lower index.  (For the largest,
 * the reference partitions at len(data) - n, the period count, so with more
 * than one period derivative its pick is numpy's partition order; callers
 * wanting that exact behaviour use the periodogram.)  PF_EUNSUPPORTED when
 * a row exceeds about 1.1e6 cells. */
int pf_ce_stats(pf_ctx* ctx, const float* const* times, const float* const* mags,
                const uint64_t* lengths, uint64_t n_curves, const float* periods,
                uint64_t n_per, const float* period_dts, uint64_t n_pdt, uint32_t n_phase,
                uint32_t n_mag, uint32_t phase_overlap, uint32_t mag_overlap, uint32_t n_top,
                int mode, float* out_stats, int64_t* out_idx, float* out_val);
int pf_aov_stats(pf_ctx* ctx, const float* const* times, const float* const* mags,
                 const uint64_t* lengths, uint64_t n_curves, const float* periods,
                 uint64_t n_per, const float* period_dts, uint64_t n_pdt, uint32_t n_phase,
                 uint32_t phase_overlap, uint32_t n_top, int mode, float* out_stats,
                 int64_t* out_idx, float* out_val);
int pf_ls_stats(pf_ctx* ctx, const float* const* times, const float* const* mags,
                const uint64_t* lengths, uint64_t n_curves, const float* periods,
                uint64_t n_per, const float* period_dts, uint64_t n_pdt, uint32_t n_top,
                int mode, float* out_stats, int64_t* out_idx, float* out_val);

/* Peak search alone on periodograms already on the host, [n_curves][flat];
 * replaces find_top_peaks_batched (rust/src/lib.rs:508-548). */
int pf_find_peaks(pf_ctx* ctx, const float* data, uint64_t n_curves,
                  uint64_t flat_len, uint32_t n_peaks, uint32_t min_distance,
                  int use_max, int64_t* out_idx, float* out_val);

/* ------------------------------------------------ device-resident callers */

/* Same computations on device memory, enqueued on `stream` (a cudaStream_t;
 * NULL = the CUDA default stream).  Curves are packed: curve c occupies
 * [offsets[c], offsets[c+1]) of d_times / d_mags; `offsets` is a HOST array
 * of n_curves + 1 entries (it drives the launch decomposition).  d_out is a
 * device array of n_curves * n_per * n_pdt floats.  The call returns once
 * the work is enqueued; it does not synchronise the stream. */
int pf_ce_dev(pf_ctx* ctx, const float* d_times, const float* d_mags,
              const int64_t* offsets, uint64_t n_curves,
              const float* d_periods, uint64_t n_per, const float* d_pdts,
              uint64_t n_pdt, uint32_t n_phase, uint32_t n_mag,
              uint32_t phase_overlap, uint32_t mag_overlap, int mode,
              float* d_out, void* stream);
int pf_aov_dev(pf_ctx* ctx, const float* d_times, const float* d_mags,
               const int64_t* offsets, uint64_t n_curves,
               const float* d_periods, uint64_t n_per, const float* d_pdts,
               uint64_t n_pdt, uint32_t n_phase, uint32_t phase_overlap,
               int mode, float* d_out, void* stream);
int pf_ls_dev(pf_ctx* ctx, const float* d_times, const float* d_mags,
              const int64_t* offsets, uint64_t n_curves,
              const float* d_periods, uint64_t n_per, const float* d_pdts,
              uint64_t n_pdt, int mode, float* d_out, void* stream);

/* Peak search on device periodograms [n_curves][flat_len]; d_out_idx /
 * d_out_val are device arrays [n_curves][n_peaks] (-1 / 0 padded). */
int pf_find_peaks_dev(pf_ctx* ctx, const float* d_data, uint64_t n_curves,
                      uint64_t flat_len, uint32_t n_peaks, uint32_t min_distance,
                      int use_max, int64_t* d_out_idx, float* d_out_val,
                      void* stream);

/* LS periodograms and their top-N peaks on device pointers, allocating
 * nothing.  No counterpart in the reference: it exists for callers that may
 * not call cudaMalloc where they need peaks -- code whose device memory is
 * owned by another allocator's pool, latency-critical paths that cannot
 * take cudaMalloc's implicit synchronisation, or fixed memory budgets.
 * Arguments are those of pf_ls_dev plus pf_find_peaks_dev's outputs (device
 * arrays [n_curves][n_peaks]); no context is used.  All scratch lives in one
 * 32 MiB device array inside the library (held by every GPU that loads it
 * until exit); a batch whose packed curves, work list and periodograms need
 * more is rejected with PF_EINVAL and a message in `err` (a caller buffer of
 * err_len bytes, may be NULL).  The first call on a device looks up the
 * array's address with that device current: make it before any stream
 * capture (the lookup is repeated once for a new CUDA context, e.g. after
 * cudaDeviceReset).  Calls share the array, so calls whose GPU work overlaps race on
 * it; order them on one stream.  Work is enqueued on `stream` (NULL = the
 * CUDA default stream) and the call returns without synchronising. */
int pf_ls_peaks_dev_noalloc(const float* d_times, const float* d_mags,
                            const int64_t* offsets, uint64_t n_curves,
                            const float* d_periods, uint64_t n_per,
                            const float* d_pdts, uint64_t n_pdt,
                            uint32_t n_peaks, uint32_t min_distance, int mode,
                            int64_t* d_out_idx, float* d_out_val, void* stream,
                            char* err, uint64_t err_len);

/* ------------------------------------------------------------ batch plans
 * No counterpart in the reference, whose drivers copy, launch and
 * synchronise per call.  A plan records the whole device pipeline for one
 * fixed batch shape -- curve packing, preparation kernels, the chosen
 * kernels' per-length-class queue launches (tuned when the plan is made),
 * and the optional top-N peak search -- as one CUDA graph, which
 * pf_plan_launch replays on any stream.  The device buffers named at
 * creation (times, magnitudes, grids, outputs) are read and written at each
 * launch, so a caller may refill the inputs in place between launches; the
 * curve offsets are copied and fixed.  Creation runs the pipeline once
 * eagerly (tuning, buffer sizing) and synchronises.  A plan owns a private
 * context; plans do not share buffers with each other or with contexts.
 * Launches of one plan must not overlap on the GPU (they share its
 * buffers).  n_peaks = 0: periodogram only.  PF_TIMING is rejected. */
#define PF_ALGO_CE 0
#define PF_ALGO_AOV 1
#define PF_ALGO_LS 2
typedef struct pf_plan pf_plan;
int pf_plan_create(int device, int algo, const float* d_times, const float* d_mags,
                   const int64_t* offsets, uint64_t n_curves, const float* d_periods,
                   uint64_t n_per, const float* d_pdts, uint64_t n_pdt, uint32_t n_phase,
                   uint32_t n_mag, uint32_t phase_overlap, uint32_t mag_overlap, int mode,
                   float* d_out, uint32_t n_peaks, uint32_t min_distance, int64_t* d_peak_idx,
                   float* d_peak_val, pf_plan** out);
int pf_plan_launch(pf_plan* plan, void* stream);
/* Last failure of this plan's launches; with NULL, of the last failed
 * pf_plan_create on this thread. */
const char* pf_plan_error(const pf_plan* plan);
void pf_plan_destroy(pf_plan* plan);
/* Number of kernel launches one pf_plan_launch replays (kernel nodes of the
 * plan's graph); 0 for NULL. */
uint64_t pf_plan_kernel_count(const pf_plan* plan);

/* Per-curve device latency of the last PF_TIMING launch on this context:
 * out_ns[c] = last end - first start (ns) over the CTAs that computed curve
 * c's periodogram; n_curves must be that launch's.  Synchronises the
 * stream that launch ran on. */
int pf_curve_latency(pf_ctx* ctx, uint64_t n_curves, double* out_ns);

/* Folded phase of every (period, time) pair as the fold kernels compute it,
 * for precision studies (no counterpart in the reference):
 * d_out[p * n + i] for device arrays d_times[n], d_periods[n_per].  mode
 * selects the fold: 0 = the reference's expression (periodfind/cuda/
 * ce.cu:140-143), PF_FOLD_EXACT, PF_FOLD_DF (turns in [-1, 1]) or PF_FOLD_F32;
 * PF_SEM_CPU selects the CPU-semantics build of it. */
int pf_fold_phase_dev(pf_ctx* ctx, int mode, const float* d_times, uint64_t n,
                      const float* d_periods, uint64_t n_per, float period_dt, float* d_out,
                      void* stream);

/* ---- Lomb-Scargle derivatives (no counterpart in the reference) ----------
 * The reference evaluates the LS power on the trial grid only
 * (periodfind/cuda/ls.cu:75-136).  These calls evaluate the same power at
 * arbitrary ANGULAR frequencies omega (radians per time unit; omega = 2 pi /
 * period) with its derivatives, for gradient-based use and for refining
 * peaks off the grid.  Inputs are CSR device arrays as in pf_ls_dev (host
 * offsets, device times / magnitudes); omega[c * omega_stride + k] (FP64,
 * stride 0 = one grid for all curves).  Outputs are [n_curves][n_freq].
 * Work is enqueued on `stream` (NULL = default stream).
 *
 * pf_ls_eval_dev: power, and where non-NULL dP/domega, d2P/domega2 and the
 * least-squares coefficients coef[2 * cell + {0, 1}] = (alpha, beta), with
 * dP/dy_i = alpha cos(omega (t_i - t0)) + beta sin(omega (t_i - t0)) and t0
 * the midpoint of the curve's time span. */
int pf_ls_eval_dev(pf_ctx* ctx, const float* d_times, const float* d_mags,
                   const int64_t* offsets, uint64_t n_curves, const double* d_omega,
                   uint64_t omega_stride, uint64_t n_freq, float* d_power, float* d_dpdw,
                   float* d_d2pdw2, float* d_coef, void* stream);

/* Backward of pf_ls_eval_dev for an upstream gradient g = dL/dpower
 * ([n_curves][n_freq]), from the forward's d_dpdw and d_coef:
 * d_grad_omega[cell] = g * dP/domega (NULL: skipped; needs d_dpdw) and
 * d_grad_mags[i] = sum_k g_k dP_k/dy_i over the curve's frequencies (NULL:
 * skipped). */
int pf_ls_backward_dev(pf_ctx* ctx, const float* d_times, const int64_t* offsets,
                       uint64_t n_curves, const double* d_omega, uint64_t omega_stride,
                       uint64_t n_freq, const float* d_grad_power, const float* d_dpdw,
                       const float* d_coef, double* d_grad_omega, float* d_grad_mags,
                       void* stream);

/* Newton refinement of LS maxima: for each (curve, k), starting at
 * d_omega0[c * n_freq + k], up to n_steps (<= 64) safeguarded Newton steps on
 * dP/domega inside [omega0 - h, omega0 + h] (h = d_half_width[cell]); writes
 * the best evaluated frequency to d_omega (may alias d_omega0) and its power
 * to d_power. */
int pf_ls_refine_dev(pf_ctx* ctx, const float* d_times, const float* d_mags,
                     const int64_t* offsets, uint64_t n_curves, const double* d_omega0,
                     const double* d_half_width, uint64_t n_freq, uint32_t n_steps,
                     double* d_omega, float* d_power, void* stream);

/* The reference's normalize=True magnitude preparation
 * (periodfind/_utils.py:39-45): out[c][i] = ((m - min) / (max - min)) * 0.999
 * + 5e-4 per curve in float32, bit-identical to numpy's evaluation of that
 * expression (one rounding per operation; NaN propagates through min / max).
 * Host arrays; several host threads for large batches.  Empty curves are
 * PF_EINVAL (numpy raises for them). */
int pf_normalize_mags(const float* const* mags, const uint64_t* lengths, uint64_t n_curves,
                      float* const* out);

/* The reference's center=True magnitude preparation
 * (periodfind/_utils.py:35-37): out[c][i] = m[i] - np.mean(m) per curve in
 * float32, bit-identical to numpy (its pairwise float32 sum, divided by the
 * length, then one subtraction per point).  Host arrays; several host
 * threads for large batches.  Empty curves are PF_EINVAL (numpy's mean of
 * an empty array is NaN with a warning; callers keep that path). */
int pf_center_mags(const float* const* mags, const uint64_t* lengths, uint64_t n_curves,
                   float* const* out);

/* The autotuner's decisions on this context, one line per (computation,
 * length class): the launch shape kept and the sample times of the fastest
 * and slowest candidates.  Writes at most len bytes (NUL-terminated) and
 * returns the number of entries. */
int pf_tuning_report(const pf_ctx* ctx, char* buf, uint64_t len);

/* Number of kernels this context has launched since creation (telemetry
 * for benchmarks: launches of the library's own kernels only). */
uint64_t pf_launch_count(const pf_ctx* ctx);

/* Device time in milliseconds of the most recent fold/statistics kernel
 * launch on this context (CUDA events around that launch), or -1. */
double pf_last_kernel_ms(const pf_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* PERIODFIND_B200_PF_H */
