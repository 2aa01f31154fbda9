/*
 * oracle.c -- CPU restatement of periodfind's batched periodogram path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity checker for the CUDA
 * library in periodfind_b200/.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / --impl reference legs of bench.py may load it.  The product
 * path never calls it and has no CPU fallback.
 *
 * It restates the reference's CPU (Rust) implementation operation for
 * operation, in IEEE single/double precision without FMA contraction
 * (build with -ffp-contract=off, no -ffast-math), so that on glibc it
 * produces the same bits the reference's Rust path produces:
 *
 *   fold       rust/src/fold.rs:13-26
 *   CE         rust/src/ce.rs:13-91
 *   AOV        rust/src/aov.rs:12-89
 *   LS         rust/src/ls.rs:15-79
 *   peaks      rust/src/peaks.rs:18-238
 *   batching   rust/src/lib.rs:31-199 (curves) and :559-677 (fused peaks)
 *
 * Two documented extensions, both off by default:
 *   - fused_tcorr=1 evaluates t - (c*t)*t with one rounding (fma), which is
 *     how nvcc contracts the same expression in periodfind/cuda/ce.cu:141,
 *     aov.cu:107,147 and ls.cu:95.  With period_dt == 0 both forms agree.
 *   - *_f64 entry points: an all-double "exact" oracle (no float rounding of
 *     the folded phase, double sums and trig) used for precision studies.
 *
 * Rust's `f32 as usize` saturates (NaN and negatives -> 0, >= 2^64 -> MAX);
 * sat_u64() restates that.  usize additions wrap (release builds).
 *
 * Parallel structure mirrors the reference: OpenMP over the flattened
 * (curve, period, pdt) space (the Rust path uses rayon par_chunks_mut over
 * curves and par_iter over the grid).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_API __attribute__((visibility("default")))
#define ORC_PI 3.14159265358979323846

/* ------------------------------------------------------------------ fold */

/* rust/src/fold.rs:13-15 */
static inline float orc_pdt_correction(float period, float period_dt) {
    return (period_dt / period) / 2.0f;
}

/* rust/src/fold.rs:22-26.  Returns the folded phase in [0, 1] as f32
 * (the f64 -> f32 rounding can produce exactly 1.0f). */
static inline float orc_fold_time(float t, float period, float pdt_corr,
                                  int fused_tcorr) {
    double td = (double)t;
    double ct = (double)pdt_corr * td;
    double t_corr = fused_tcorr ? fma(-ct, td, td) : td - ct * td;
    double ratio = t_corr / (double)period;
    return (float)fabs(ratio - floor(ratio));
}

/* Saturating f32 -> u64 cast with Rust `as usize` semantics. */
static inline uint64_t sat_u64(float x) {
    if (!(x > 0.0f)) return 0;
    if (x >= 18446744073709551616.0f) return UINT64_MAX;
    return (uint64_t)x;
}

static void set_threads(int n_threads) {
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#else
    (void)n_threads;
#endif
}

/* ------------------------------------------------------------------- CE */

/* One (period, pdt) cell of rust/src/ce.rs:39-116.  `hist` is scratch of
 * num_phase*num_mag u32.  If `counts_out` is non-NULL the raw histogram is
 * copied there (test hook for bin-occupancy comparisons). */
static float orc_ce_cell(const float* times, const float* mags, uint64_t length,
                         float period, float period_dt, uint32_t num_phase,
                         uint32_t num_mag, uint32_t phase_overlap,
                         uint32_t mag_overlap, uint32_t* hist,
                         uint32_t* counts_out, int fused_tcorr) {
    const uint64_t num_bins = (uint64_t)num_phase * num_mag;
    const float phase_bin_size = 1.0f / (float)num_phase;
    const float mag_bin_size = 1.0f / (float)num_mag;
    const float norm_divisor =
        (float)(length * (uint64_t)phase_overlap * (uint64_t)mag_overlap);
    const float pdt_corr = orc_pdt_correction(period, period_dt);

    memset(hist, 0, num_bins * sizeof(uint32_t));
    for (uint64_t i = 0; i < length; i++) {
        float folded = orc_fold_time(times[i], period, pdt_corr, fused_tcorr);
        uint64_t phase_bin = sat_u64(folded / phase_bin_size);
        uint64_t mag_bin = sat_u64(mags[i] / mag_bin_size);
        for (uint64_t po = 0; po < phase_overlap; po++) {
            for (uint64_t mo = 0; mo < mag_overlap; mo++) {
                uint64_t pb = (phase_bin + po) % num_phase;
                uint64_t mb = (mag_bin + mo) % num_mag;
                hist[pb * num_mag + mb] += 1;
            }
        }
    }
    if (counts_out) memcpy(counts_out, hist, num_bins * sizeof(uint32_t));

    /* rust/src/ce.rs:91-112: normalise, then sum p_ij ln(p_j / p_ij). */
    float ce = 0.0f;
    for (uint32_t j = 0; j < num_phase; j++) {
        float p_j = 0.0f;
        for (uint32_t i = 0; i < num_mag; i++)
            p_j += (float)hist[j * num_mag + i] / norm_divisor;
        for (uint32_t i = 0; i < num_mag; i++) {
            float p_ij = (float)hist[j * num_mag + i] / norm_divisor;
            if (p_ij != 0.0f) ce += p_ij * logf(p_j / p_ij);
        }
    }
    return ce;
}

/* Batched CE (rust/src/lib.rs:31-88).  Curves are given CSR style:
 * curve c occupies [offsets[c], offsets[c+1]) of times/mags.  Output is
 * out[c][period][pdt] (C order). */
ORC_API void orc_ce_batched(const float* times, const float* mags,
                            const int64_t* offsets, int64_t n_curves,
                            const float* periods, int64_t n_per,
                            const float* pdts, int64_t n_pdt,
                            uint32_t num_phase, uint32_t num_mag,
                            uint32_t phase_overlap, uint32_t mag_overlap,
                            int fused_tcorr, int n_threads, float* out) {
    set_threads(n_threads);
    const int64_t per_curve = n_per * n_pdt;
    const int64_t total = n_curves * per_curve;
    if (total == 0) return;
#pragma omp parallel
    {
        uint32_t* hist =
            (uint32_t*)malloc((size_t)num_phase * num_mag * sizeof(uint32_t));
#pragma omp for schedule(dynamic, 64)
        for (int64_t k = 0; k < total; k++) {
            int64_t c = k / per_curve, g = k % per_curve;
            int64_t p = g / n_pdt, d = g % n_pdt;
            const int64_t o = offsets[c];
            out[k] = orc_ce_cell(times + o, mags + o,
                                 (uint64_t)(offsets[c + 1] - o), periods[p],
                                 pdts[d], num_phase, num_mag, phase_overlap,
                                 mag_overlap, hist, NULL, fused_tcorr);
        }
        free(hist);
    }
}

/* Test hook: raw CE histogram for one curve and one (period, pdt). */
ORC_API float orc_ce_counts(const float* times, const float* mags,
                            int64_t length, float period, float period_dt,
                            uint32_t num_phase, uint32_t num_mag,
                            uint32_t phase_overlap, uint32_t mag_overlap,
                            int fused_tcorr, uint32_t* counts_out) {
    uint32_t* hist =
        (uint32_t*)malloc((size_t)num_phase * num_mag * sizeof(uint32_t));
    float v = orc_ce_cell(times, mags, (uint64_t)length, period, period_dt,
                          num_phase, num_mag, phase_overlap, mag_overlap, hist,
                          counts_out, fused_tcorr);
    free(hist);
    return v;
}

/* ------------------------------------------------------------------ FPW */

/* rust/src/fpw.rs:12-66 for one curve and one (period, pdt): inverse
 * variances w = 1 / err^2 and w * m (computed once per curve by the caller),
 * per bin V = sum w and Y = sum w * m in point order, then
 * sum over bins with V > 0 of Y^2 / (2 V), all in f32. */
static float orc_fpw_cell(const float* times, const float* iv, const float* ivy,
                          uint64_t length, float period, float period_dt,
                          uint32_t num_bins, float* vt, float* yt) {
    const float pdt_corr = orc_pdt_correction(period, period_dt);
    for (uint32_t k = 0; k < num_bins; k++) vt[k] = yt[k] = 0.0f;
    for (uint64_t i = 0; i < length; i++) {
        const float phase = orc_fold_time(times[i], period, pdt_corr, 0);
        uint64_t bin = sat_u64(phase * (float)num_bins);
        if (bin > num_bins - 1) bin = num_bins - 1;
        vt[bin] += iv[i];
        yt[bin] += ivy[i];
    }
    float delta_chi = 0.0f;
    for (uint32_t k = 0; k < num_bins; k++)
        if (vt[k] > 0.0f) delta_chi += yt[k] * yt[k] / (2.0f * vt[k]);
    return delta_chi;
}

/* rust/src/lib.rs:202-256 (calc_fpw_batched): errs NULL means err = 1. */
ORC_API void orc_fpw_batched(const float* times, const float* mags, const float* errs,
                             const int64_t* offsets, int64_t n_curves,
                             const float* periods, int64_t n_per,
                             const float* pdts, int64_t n_pdt, uint32_t num_bins,
                             int n_threads, float* out) {
    set_threads(n_threads);
    const int64_t n_pts = n_curves > 0 ? offsets[n_curves] : 0;
    float* iv = (float*)malloc((size_t)(n_pts > 0 ? n_pts : 1) * sizeof(float));
    float* ivy = (float*)malloc((size_t)(n_pts > 0 ? n_pts : 1) * sizeof(float));
    for (int64_t i = 0; i < n_pts; i++) {
        const float e = errs ? errs[i] : 1.0f;
        iv[i] = 1.0f / (e * e);
        ivy[i] = iv[i] * mags[i];
    }
    const int64_t per_curve = n_per * n_pdt;
    const int64_t total = n_curves * per_curve;
#pragma omp parallel
    {
        float* vt = (float*)malloc((size_t)num_bins * sizeof(float));
        float* yt = (float*)malloc((size_t)num_bins * sizeof(float));
#pragma omp for schedule(dynamic, 64)
        for (int64_t k = 0; k < total; k++) {
            int64_t c = k / per_curve, g = k % per_curve;
            int64_t p = g / n_pdt, d = g % n_pdt;
            const int64_t o = offsets[c];
            out[k] = orc_fpw_cell(times + o, iv + o, ivy + o, (uint64_t)(offsets[c + 1] - o),
                                  periods[p], pdts[d], num_bins, vt, yt);
        }
        free(vt);
        free(yt);
    }
    free(iv);
    free(ivy);
}

/* ------------------------------------------------------------------ BLS */

/* rust/src/bls.rs:19-134 for one curve and one (period, pdt): bins of w and
 * w * (m - mean) (the caller's arrays), prefix sums, and the best
 * s^2 / (r (W - r)) over windows of nb_min .. nb_max bins, all in f32. */
static float orc_bls_cell(const float* times, const float* iv, const float* iyw,
                          uint64_t length, float period, float period_dt, uint32_t num_bins,
                          uint64_t nb_min, uint64_t nb_max, float* wb, float* yb,
                          float* wp, float* yp) {
    const float pdt_corr = orc_pdt_correction(period, period_dt);
    for (uint32_t k = 0; k < num_bins; k++) wb[k] = yb[k] = 0.0f;
    for (uint64_t i = 0; i < length; i++) {
        const float phase = orc_fold_time(times[i], period, pdt_corr, 0);
        uint64_t bin = sat_u64(phase * (float)num_bins);
        if (bin > num_bins - 1) bin = num_bins - 1;
        wb[bin] += iv[i];
        yb[bin] += iyw[i];
    }
    wp[0] = 0.0f;
    yp[0] = 0.0f;
    for (uint32_t k = 0; k < num_bins; k++) {
        wp[k + 1] = wp[k] + wb[k];
        yp[k + 1] = yp[k] + yb[k];
    }
    const float w_total = wp[num_bins];
    if (w_total <= 0.0f) return 0.0f;
    float best = 0.0f;
    for (uint64_t nb = nb_min; nb <= nb_max; nb++) {
        for (uint64_t phi = 0; phi < num_bins; phi++) {
            const uint64_t end = phi + nb;
            float r, s;
            if (end <= num_bins) {
                r = wp[end] - wp[phi];
                s = yp[end] - yp[phi];
            } else {
                const uint64_t wrap = end - num_bins;
                r = (wp[num_bins] - wp[phi]) + wp[wrap];
                s = (yp[num_bins] - yp[phi]) + yp[wrap];
            }
            const float r_frac = r / w_total;
            if (r_frac > 0.0f && r_frac < 1.0f) {
                const float v = (s * s) / (r * (w_total - r));
                if (v > best) best = v;
            }
        }
    }
    return best;
}

/* rust/src/lib.rs:264-322 (calc_bls_batched): errs NULL means err = 1. */
ORC_API void orc_bls_batched(const float* times, const float* mags, const float* errs,
                             const int64_t* offsets, int64_t n_curves,
                             const float* periods, int64_t n_per,
                             const float* pdts, int64_t n_pdt, uint32_t num_bins,
                             float qmin, float qmax, int n_threads, float* out) {
    set_threads(n_threads);
    const int64_t n_pts = n_curves > 0 ? offsets[n_curves] : 0;
    float* iv = (float*)malloc((size_t)(n_pts > 0 ? n_pts : 1) * sizeof(float));
    float* iyw = (float*)malloc((size_t)(n_pts > 0 ? n_pts : 1) * sizeof(float));
    for (int64_t c = 0; c < n_curves; c++) {
        float total_w = 0.0f, total_wy = 0.0f;
        for (int64_t i = offsets[c]; i < offsets[c + 1]; i++) {
            const float e = errs ? errs[i] : 1.0f;
            iv[i] = 1.0f / (e * e);
            total_w += iv[i];
        }
        for (int64_t i = offsets[c]; i < offsets[c + 1]; i++) total_wy += iv[i] * mags[i];
        const float mean_y = total_w > 0.0f ? total_wy / total_w : 0.0f;
        for (int64_t i = offsets[c]; i < offsets[c + 1]; i++) iyw[i] = iv[i] * (mags[i] - mean_y);
    }
    /* bls.rs:51-52 with Rust's saturating casts */
    const uint64_t lo = sat_u64(floorf(qmin * (float)num_bins));
    const uint64_t hi = sat_u64(ceilf(qmax * (float)num_bins));
    const uint64_t nb_min = lo > 1 ? lo : 1;
    const uint64_t nb_max = hi < (uint64_t)num_bins - 1 ? hi : (uint64_t)num_bins - 1;
    const int64_t per_curve = n_per * n_pdt;
    const int64_t total = n_curves * per_curve;
#pragma omp parallel
    {
        float* wb = (float*)malloc((size_t)num_bins * sizeof(float));
        float* yb = (float*)malloc((size_t)num_bins * sizeof(float));
        float* wp = (float*)malloc((size_t)(num_bins + 1) * sizeof(float));
        float* yp = (float*)malloc((size_t)(num_bins + 1) * sizeof(float));
#pragma omp for schedule(dynamic, 64)
        for (int64_t k = 0; k < total; k++) {
            int64_t c = k / per_curve, g = k % per_curve;
            int64_t p = g / n_pdt, d = g % n_pdt;
            const int64_t o = offsets[c];
            out[k] = orc_bls_cell(times + o, iv + o, iyw + o, (uint64_t)(offsets[c + 1] - o),
                                  periods[p], pdts[d], num_bins, nb_min, nb_max, wb, yb, wp, yp);
        }
        free(wb);
        free(yb);
        free(wp);
        free(yp);
    }
    free(iv);
    free(iyw);
}

/* ------------------------------------------------------------------ AOV */

typedef struct {
    uint32_t* count;
    float* sums;
    float* sq_sums;
} aov_scratch;

/* rust/src/aov.rs:27: sequential f32 sum, then divide. */
static float orc_array_mean(const float* mags, uint64_t length) {
    float s = 0.0f;
    for (uint64_t i = 0; i < length; i++) s += mags[i];
    return s / (float)length;
}

/* One (period, pdt) cell of rust/src/aov.rs:12-89. */
static float orc_aov_cell(const float* times, const float* mags,
                          uint64_t length, float avg, float period,
                          float period_dt, uint32_t num_bins,
                          uint32_t num_overlap, aov_scratch* s,
                          uint32_t* counts_out, int fused_tcorr) {
    const float bin_size = 1.0f / (float)num_bins;
    const float pdt_corr = orc_pdt_correction(period, period_dt);
    memset(s->count, 0, num_bins * sizeof(uint32_t));
    memset(s->sums, 0, num_bins * sizeof(float));
    memset(s->sq_sums, 0, num_bins * sizeof(float));
    for (uint64_t i = 0; i < length; i++) {
        float folded = orc_fold_time(times[i], period, pdt_corr, fused_tcorr);
        uint64_t bin = sat_u64(folded / bin_size);
        float mag = mags[i];
        for (uint64_t o = 0; o < num_overlap; o++) {
            uint64_t b = (bin + o) % num_bins;
            s->count[b] += 1;
            s->sums[b] += mag;
            s->sq_sums[b] += mag * mag;
        }
    }
    if (counts_out) memcpy(counts_out, s->count, num_bins * sizeof(uint32_t));

    float s1 = 0.0f, s2 = 0.0f;
    for (uint32_t b = 0; b < num_bins; b++) {
        float n = (float)s->count[b];
        if (n != 0.0f) {
            float aux = s->sums[b] / n;
            float residual = aux - avg;
            s1 += n * residual * residual;
            s2 += s->sq_sums[b] - n * aux * aux;
        }
    }
    if (s2 == 0.0f) return 0.0f;
    return (((float)length - (float)num_bins) / ((float)num_bins - 1.0f)) *
           (s1 / s2);
}

ORC_API void orc_aov_batched(const float* times, const float* mags,
                             const int64_t* offsets, int64_t n_curves,
                             const float* periods, int64_t n_per,
                             const float* pdts, int64_t n_pdt,
                             uint32_t num_bins, uint32_t num_overlap,
                             int fused_tcorr, int n_threads, float* out) {
    set_threads(n_threads);
    const int64_t per_curve = n_per * n_pdt;
    const int64_t total = n_curves * per_curve;
    if (total == 0) return;
    float* avgs = (float*)malloc((size_t)(n_curves > 0 ? n_curves : 1) *
                                 sizeof(float));
    for (int64_t c = 0; c < n_curves; c++)
        avgs[c] = orc_array_mean(mags + offsets[c],
                                 (uint64_t)(offsets[c + 1] - offsets[c]));
#pragma omp parallel
    {
        aov_scratch s;
        s.count = (uint32_t*)malloc(num_bins * sizeof(uint32_t));
        s.sums = (float*)malloc(num_bins * sizeof(float));
        s.sq_sums = (float*)malloc(num_bins * sizeof(float));
#pragma omp for schedule(dynamic, 64)
        for (int64_t k = 0; k < total; k++) {
            int64_t c = k / per_curve, g = k % per_curve;
            int64_t p = g / n_pdt, d = g % n_pdt;
            const int64_t o = offsets[c];
            out[k] = orc_aov_cell(times + o, mags + o,
                                  (uint64_t)(offsets[c + 1] - o), avgs[c],
                                  periods[p], pdts[d], num_bins, num_overlap,
                                  &s, NULL, fused_tcorr);
        }
        free(s.count);
        free(s.sums);
        free(s.sq_sums);
    }
    free(avgs);
}

ORC_API float orc_aov_counts(const float* times, const float* mags,
                             int64_t length, float period, float period_dt,
                             uint32_t num_bins, uint32_t num_overlap,
                             int fused_tcorr, uint32_t* counts_out) {
    aov_scratch s;
    s.count = (uint32_t*)malloc(num_bins * sizeof(uint32_t));
    s.sums = (float*)malloc(num_bins * sizeof(float));
    s.sq_sums = (float*)malloc(num_bins * sizeof(float));
    float avg = orc_array_mean(mags, (uint64_t)length);
    float v = orc_aov_cell(times, mags, (uint64_t)length, avg, period,
                           period_dt, num_bins, num_overlap, &s, counts_out,
                           fused_tcorr);
    free(s.count);
    free(s.sums);
    free(s.sq_sums);
    return v;
}

/* ------------------------------------------------------------------- LS */

/* rust/src/ls.rs:15-79 for one (period, pdt) cell. */
static float orc_ls_cell(const float* times, const float* mags,
                         uint64_t length, float period, float period_dt,
                         int fused_tcorr) {
    const float two_pi = 2.0f * (float)ORC_PI; /* ls.rs:13 (f32 PI) */
    const float pdt_corr = orc_pdt_correction(period, period_dt);
    float mag_cos = 0.0f, mag_sin = 0.0f, cos_cos = 0.0f, cos_sin = 0.0f;
    for (uint64_t i = 0; i < length; i++) {
        float folded = orc_fold_time(times[i], period, pdt_corr, fused_tcorr);
        float angle = two_pi * folded;
        float sin_val = sinf(angle), cos_val = cosf(angle);
        mag_cos += mags[i] * cos_val;
        mag_sin += mags[i] * sin_val;
        cos_cos += cos_val * cos_val;
        cos_sin += cos_val * sin_val;
    }
    float sin_sin = (float)length - cos_cos;
    float tau_angle = 0.5f * atan2f(2.0f * cos_sin, cos_cos - sin_sin);
    float sin_tau = sinf(tau_angle), cos_tau = cosf(tau_angle);
    float v;
    v = cos_tau * mag_cos + sin_tau * mag_sin;
    float num_l = v * v;
    v = cos_tau * mag_sin - sin_tau * mag_cos;
    float num_r = v * v;
    float den_l = cos_tau * cos_tau * cos_cos +
                  2.0f * cos_tau * sin_tau * cos_sin +
                  sin_tau * sin_tau * sin_sin;
    float den_r = cos_tau * cos_tau * sin_sin -
                  2.0f * cos_tau * sin_tau * cos_sin +
                  sin_tau * sin_tau * cos_cos;
    if (den_l == 0.0f || den_r == 0.0f) return 0.0f;
    return 0.5f * (num_l / den_l + num_r / den_r);
}

ORC_API void orc_ls_batched(const float* times, const float* mags,
                            const int64_t* offsets, int64_t n_curves,
                            const float* periods, int64_t n_per,
                            const float* pdts, int64_t n_pdt, int fused_tcorr,
                            int n_threads, float* out) {
    set_threads(n_threads);
    const int64_t per_curve = n_per * n_pdt;
    const int64_t total = n_curves * per_curve;
    if (total == 0) return;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t k = 0; k < total; k++) {
        int64_t c = k / per_curve, g = k % per_curve;
        int64_t p = g / n_pdt, d = g % n_pdt;
        const int64_t o = offsets[c];
        out[k] = orc_ls_cell(times + o, mags + o,
                             (uint64_t)(offsets[c + 1] - o), periods[p],
                             pdts[d], fused_tcorr);
    }
}

/* --------------------------------------------------- FP64 exact oracle */

/* AOV with the reference's bins (f32 fold, IEEE bin division, as
 * rust/src/aov.rs:170-181) but every sum and the statistic in double: the
 * value the f32 accumulation approximates. */
ORC_API void orc_aov_batched_f64(const float* times, const float* mags,
                                 const int64_t* offsets, int64_t n_curves,
                                 const float* periods, int64_t n_per,
                                 const float* pdts, int64_t n_pdt,
                                 uint32_t num_bins, uint32_t num_overlap,
                                 int fused_tcorr, int n_threads, double* out) {
    set_threads(n_threads);
    const int64_t per_curve = n_per * n_pdt;
    const int64_t total = n_curves * per_curve;
    if (total == 0) return;
#pragma omp parallel
    {
        double* cnt = (double*)malloc(num_bins * sizeof(double));
        double* sum = (double*)malloc(num_bins * sizeof(double));
        double* sq = (double*)malloc(num_bins * sizeof(double));
#pragma omp for schedule(dynamic, 64)
        for (int64_t k = 0; k < total; k++) {
            int64_t c = k / per_curve, g = k % per_curve;
            int64_t p = g / n_pdt, d = g % n_pdt;
            const int64_t o = offsets[c];
            const uint64_t length = (uint64_t)(offsets[c + 1] - o);
            const float* t = times + o;
            const float* m = mags + o;
            const float bin_size = 1.0f / (float)num_bins;
            const float pdt_corr = orc_pdt_correction(periods[p], pdts[d]);
            double tot = 0.0;
            for (uint64_t i = 0; i < length; i++) tot += m[i];
            const double avg = length ? tot / (double)length : 0.0;
            memset(cnt, 0, num_bins * sizeof(double));
            memset(sum, 0, num_bins * sizeof(double));
            memset(sq, 0, num_bins * sizeof(double));
            for (uint64_t i = 0; i < length; i++) {
                float folded = orc_fold_time(t[i], periods[p], pdt_corr, fused_tcorr);
                uint64_t bin = sat_u64(folded / bin_size);
                for (uint64_t ov = 0; ov < num_overlap; ov++) {
                    uint64_t b = (bin + ov) % num_bins;
                    cnt[b] += 1.0;
                    sum[b] += (double)m[i];
                    sq[b] += (double)m[i] * (double)m[i];
                }
            }
            double s1 = 0.0, s2 = 0.0;
            for (uint32_t b = 0; b < num_bins; b++) {
                if (cnt[b] != 0.0) {
                    double mu = sum[b] / cnt[b];
                    s1 += cnt[b] * (mu - avg) * (mu - avg);
                    s2 += sq[b] - cnt[b] * mu * mu;
                }
            }
            out[k] = (s2 == 0.0) ? 0.0
                     : (((double)length - (double)num_bins) / ((double)num_bins - 1.0)) * (s1 / s2);
        }
        free(cnt);
        free(sum);
        free(sq);
    }
}


/* Same statistic as orc_ls_cell with every step in double and no float
 * rounding of the folded phase: the reference value for precision studies.
 * The trial frequency is the f32 period promoted to double. */
static double orc_ls_cell_f64(const float* times, const float* mags,
                              uint64_t length, double period, double period_dt) {
    const double two_pi = 2.0 * ORC_PI;
    const double pdt_corr = (period_dt / period) / 2.0;
    double mc = 0, ms = 0, cc = 0, cs = 0;
    for (uint64_t i = 0; i < length; i++) {
        double t = (double)times[i];
        double r = (t - pdt_corr * t * t) / period;
        double ph = r - floor(r);
        double s = sin(two_pi * ph), c = cos(two_pi * ph);
        mc += mags[i] * c;
        ms += mags[i] * s;
        cc += c * c;
        cs += c * s;
    }
    double ss = (double)length - cc;
    double tau = 0.5 * atan2(2.0 * cs, cc - ss);
    double st = sin(tau), ct = cos(tau);
    double a = ct * mc + st * ms, b = ct * ms - st * mc;
    double dl = ct * ct * cc + 2.0 * ct * st * cs + st * st * ss;
    double dr = ct * ct * ss - 2.0 * ct * st * cs + st * st * cc;
    if (dl == 0.0 || dr == 0.0) return 0.0;
    return 0.5 * (a * a / dl + b * b / dr);
}

ORC_API void orc_ls_batched_f64(const float* times, const float* mags,
                                const int64_t* offsets, int64_t n_curves,
                                const double* periods, int64_t n_per,
                                const double* pdts, int64_t n_pdt,
                                int n_threads, double* out) {
    set_threads(n_threads);
    const int64_t per_curve = n_per * n_pdt;
    const int64_t total = n_curves * per_curve;
    if (total == 0) return;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t k = 0; k < total; k++) {
        int64_t c = k / per_curve, g = k % per_curve;
        int64_t p = g / n_pdt, d = g % n_pdt;
        const int64_t o = offsets[c];
        out[k] = orc_ls_cell_f64(times + o, mags + o,
                                 (uint64_t)(offsets[c + 1] - o), periods[p],
                                 pdts[d]);
    }
}

/* Exact folded phase (double, no float rounding) for precision studies:
 * out[p * n + i] = frac((t_i - c t_i^2) / P_p) with c = (pdt/P)/2 in double. */
ORC_API void orc_phase_f64(const float* times, int64_t n, const double* periods,
                           int64_t n_per, double period_dt, int n_threads,
                           double* out) {
    set_threads(n_threads);
#pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < n_per; p++) {
        double P = periods[p];
        double c = (period_dt / P) / 2.0;
        for (int64_t i = 0; i < n; i++) {
            double t = (double)times[i];
            double r = (t - c * t * t) / P;
            out[p * n + i] = r - floor(r);
        }
    }
}

/* ------------------------------------------------------ LS derivatives */

/* The LS power as a function of angular frequency w, with its first and
 * second w-derivatives, in FP64.  No counterpart in the reference (which
 * evaluates the power on the trial grid only, rust/src/ls.rs:231-276); the
 * power itself equals orc_ls_cell_f64 (the reference's tau expression,
 * ls.rs:253-275) because tau only diagonalises the 2x2 normal matrix:
 *   P = 0.5 v^T M^-1 v,  v = (C, S),  M = [[CC, CS], [CS, SS]],  w = M^-1 v.
 * Times are measured from the midpoint t0 of the curve's time span, the
 * convention under which (alpha, beta) = M^-1 v are reported. */
static double ls_t0(const float* t, uint64_t n) {
    if (n == 0) return 0.0;
    float lo = t[0], hi = t[0];
    for (uint64_t i = 1; i < n; i++) {
        if (t[i] < lo) lo = t[i];
        if (t[i] > hi) hi = t[i];
    }
    return 0.5 * ((double)lo + (double)hi);
}

static void ls_deriv_cell_f64(const float* t, const float* y, uint64_t n, double w,
                              double out[5]) {
    const double t0 = ls_t0(t, n);
    double C = 0, S = 0, CC = 0, CS = 0, C1 = 0, S1 = 0, CC1 = 0, CS1 = 0;
    double C2 = 0, S2 = 0, CC2 = 0, CS2 = 0;
    for (uint64_t i = 0; i < n; i++) {
        const double x = (double)t[i] - t0, yy = (double)y[i];
        const double th = w * x;
        const double s = sin(th), c = cos(th);
        const double s2 = sin(2.0 * th), c2 = cos(2.0 * th);
        C += yy * c;
        S += yy * s;
        CC += c * c;
        CS += c * s;
        C1 -= yy * x * s;
        S1 += yy * x * c;
        CC1 -= x * s2;
        CS1 += x * c2;
        C2 -= yy * x * x * c;
        S2 -= yy * x * x * s;
        CC2 -= 2.0 * x * x * c2;
        CS2 -= 2.0 * x * x * s2;
    }
    const double SS = (double)n - CC;
    const double det = CC * SS - CS * CS;
    for (int k = 0; k < 5; k++) out[k] = 0.0;
    if (!(det > 1e-6 * CC * SS)) return; /* singular M: power 0, as the device */
    const double al = (SS * C - CS * S) / det, be = (CC * S - CS * C) / det;
    const double u0 = C1 - (CC1 * al + CS1 * be), u1 = S1 - (CS1 * al - CC1 * be);
    out[0] = 0.5 * (al * C + be * S);
    out[1] = al * C1 + be * S1 - 0.5 * ((al * al - be * be) * CC1 + 2.0 * al * be * CS1);
    out[2] = (SS * u0 * u0 - 2.0 * CS * u0 * u1 + CC * u1 * u1) / det + al * C2 + be * S2 -
             0.5 * ((al * al - be * be) * CC2 + 2.0 * al * be * CS2);
    out[3] = al;
    out[4] = be;
}

/* out[cell * 5 + {0..4}] = (P, dP/dw, d2P/dw2, alpha, beta) for
 * w = omega[c * omega_stride + k]. */
ORC_API void orc_ls_derivs_f64(const float* times, const float* mags, const int64_t* offsets,
                               int64_t n_curves, const double* omega, int64_t omega_stride,
                               int64_t n_freq, int n_threads, double* out) {
    set_threads(n_threads);
    const int64_t total = n_curves * n_freq;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t cell = 0; cell < total; cell++) {
        const int64_t c = cell / n_freq, k = cell % n_freq;
        const int64_t o = offsets[c];
        ls_deriv_cell_f64(times + o, mags + o, (uint64_t)(offsets[c + 1] - o),
                          omega[c * omega_stride + k], out + 5 * cell);
    }
}

/* dL/dy_i = sum_k (g alpha)_k cos(w_k (t_i - t0)) + (g beta)_k sin(...),
 * gcoef[cell * 2 + {0, 1}] = upstream gradient times (alpha, beta). */
ORC_API void orc_ls_grad_mags_f64(const float* times, const int64_t* offsets, int64_t n_curves,
                                  const double* omega, int64_t omega_stride, int64_t n_freq,
                                  const double* gcoef, int n_threads, double* out) {
    set_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < n_curves; c++) {
        const int64_t o = offsets[c];
        const uint64_t n = (uint64_t)(offsets[c + 1] - o);
        const double t0 = ls_t0(times + o, n);
        for (uint64_t i = 0; i < n; i++) {
            const double x = (double)times[o + i] - t0;
            double acc = 0.0;
            for (int64_t k = 0; k < n_freq; k++) {
                const double th = omega[c * omega_stride + k] * x;
                acc += gcoef[2 * (c * n_freq + k)] * cos(th) +
                       gcoef[2 * (c * n_freq + k) + 1] * sin(th);
            }
            out[o + i] = acc;
        }
    }
}

/* Safeguarded Newton toward the LS maximum, the control flow the device
 * refinement follows: n_steps updates inside [w0 - h, w0 + h]; Newton where
 * d2P/dw2 < 0, else a quarter-bracket step uphill; n_steps + 1 evaluations.
 * The last iterate is returned unless its power is more than 1e-5 (relative)
 * below the best evaluated one, which is returned then. */
ORC_API void orc_ls_refine_f64(const float* times, const float* mags, const int64_t* offsets,
                               int64_t n_curves, const double* omega0,
                               const double* half_width, int64_t n_freq, int n_steps,
                               int n_threads, double* omega_out, double* power_out) {
    set_threads(n_threads);
    const int64_t total = n_curves * n_freq;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t cell = 0; cell < total; cell++) {
        const int64_t c = cell / n_freq;
        const int64_t o = offsets[c];
        const uint64_t n = (uint64_t)(offsets[c + 1] - o);
        double w = omega0[cell];
        const double hw = half_width[cell], lo = w - hw, hi = w + hw;
        double best_w = w, best_p = -1.0, last_w = w, last_p = -1.0;
        for (int e = 0; e <= n_steps; e++) {
            double d[5];
            ls_deriv_cell_f64(times + o, mags + o, n, w, d);
            last_p = d[0];
            last_w = w;
            if (d[0] > best_p) {
                best_p = d[0];
                best_w = w;
            }
            if (e < n_steps) {
                double step = (d[2] < 0.0) ? -d[1] / d[2] : ((d[1] > 0.0) ? 0.25 * hw : -0.25 * hw);
                w = fmin(fmax(w + step, lo), hi);
            }
        }
        /* the last iterate unless its power is clearly below the best */
        const int keep_last = last_p >= best_p * (1.0 - 1e-5);
        omega_out[cell] = keep_last ? last_w : best_w;
        const double pw = keep_last ? last_p : best_p;
        power_out[cell] = pw > 0.0 ? pw : 0.0;
    }
}

/* The reference's tau expression (rust/src/ls.rs:253-275) in FP64 with FP64
 * magnitudes, at angular frequency w: the target of finite-difference
 * gradient checks. */
ORC_API double orc_ls_power_tau_f64(const double* t, const double* y, int64_t n, double w) {
    double mc = 0, ms = 0, cc = 0, cs = 0;
    for (int64_t i = 0; i < n; i++) {
        const double s = sin(w * t[i]), c = cos(w * t[i]);
        mc += y[i] * c;
        ms += y[i] * s;
        cc += c * c;
        cs += c * s;
    }
    const double ss = (double)n - cc;
    const double tau = 0.5 * atan2(2.0 * cs, cc - ss);
    const double st = sin(tau), ct = cos(tau);
    const double a = ct * mc + st * ms, b = ct * ms - st * mc;
    const double dl = ct * ct * cc + 2.0 * ct * st * cs + st * st * ss;
    const double dr = ct * ct * ss - 2.0 * ct * st * cs + st * st * cc;
    if (dl == 0.0 || dr == 0.0) return 0.0;
    return 0.5 * (a * a / dl + b * b / dr);
}

/* ---------------------------------------------------------------- peaks */

/* Streaming greedy top-N peak finder, rust/src/peaks.rs:18-218, applied in
 * one chunk (find_top_peaks, peaks.rs:228-238). */
typedef struct {
    int64_t* indices;
    float* values;
    uint64_t count;
    uint64_t n_peaks;
    uint64_t min_distance;
    int use_max;
    int64_t cand_idx;
    float cand_val;
    int has_cand;
    uint64_t dist;
} peak_state;

static inline int pk_better(const peak_state* s, float a, float b) {
    return s->use_max ? (a > b) : (a < b);
}
static inline int pk_is_peak(const peak_state* s, float l, float v, float r) {
    return s->use_max ? (v > l && v > r) : (v < l && v < r);
}
static inline float pk_threshold(const peak_state* s) {
    if (s->count < s->n_peaks) return s->use_max ? -INFINITY : INFINITY;
    return s->values[s->count - 1];
}
static void pk_insert(peak_state* s, int64_t idx, float val) {
    uint64_t i;
    if (s->count < s->n_peaks) {
        i = s->count++;
        s->indices[i] = idx;
        s->values[i] = val;
    } else if (pk_better(s, val, s->values[s->count - 1])) {
        i = s->count - 1;
        s->indices[i] = idx;
        s->values[i] = val;
    } else {
        return;
    }
    while (i > 0 && pk_better(s, s->values[i], s->values[i - 1])) {
        float tv = s->values[i];
        s->values[i] = s->values[i - 1];
        s->values[i - 1] = tv;
        int64_t ti = s->indices[i];
        s->indices[i] = s->indices[i - 1];
        s->indices[i - 1] = ti;
        i--;
    }
}
static inline void pk_try_promote(peak_state* s) {
    if (s->has_cand && pk_better(s, s->cand_val, pk_threshold(s)))
        pk_insert(s, s->cand_idx, s->cand_val);
    s->has_cand = 0;
    s->dist = 0;
}
static inline void pk_feed(peak_state* s, float v, float l, float r,
                           int64_t idx) {
    if (pk_is_peak(s, l, v, r) && pk_better(s, v, pk_threshold(s))) {
        if (!s->has_cand || pk_better(s, v, s->cand_val)) {
            s->cand_idx = idx;
            s->cand_val = v;
            s->has_cand = 1;
            s->dist = 0;
        }
    }
    if (s->has_cand) {
        s->dist += 1;
        if (s->dist >= s->min_distance) pk_try_promote(s);
    }
}

/* find_top_peaks: returns the number of peaks written (<= n_peaks). */
ORC_API int64_t orc_find_top_peaks(const float* data, int64_t n,
                                   int64_t n_peaks, int64_t min_distance,
                                   int use_max, int64_t* out_idx,
                                   float* out_val) {
    peak_state s;
    memset(&s, 0, sizeof(s));
    s.indices = out_idx;
    s.values = out_val;
    s.n_peaks = (uint64_t)n_peaks;
    s.min_distance = (uint64_t)min_distance;
    s.use_max = use_max;
    s.cand_idx = -1;
    s.cand_val = use_max ? -INFINITY : INFINITY;
    if (n_peaks <= 0) return 0;
    for (int64_t i = 0; i < n_peaks; i++) {
        out_idx[i] = 0;
        out_val[i] = use_max ? -INFINITY : INFINITY;
    }
    /* process_chunk with has_prev == false (peaks.rs:166-204): interior
     * points 1 .. n-2 only. */
    for (int64_t i = 1; i + 1 < n; i++)
        pk_feed(&s, data[i], data[i - 1], data[i + 1], i);
    pk_try_promote(&s); /* finalize */
    return (int64_t)s.count;
}

/* Batched form (rust/src/lib.rs:508-548): data is [n_curves][flat_len];
 * outputs are [n_curves][n_peaks], idx padded with -1, val padded with 0. */
ORC_API void orc_find_top_peaks_batched(const float* data, int64_t n_curves,
                                        int64_t flat_len, int64_t n_peaks,
                                        int64_t min_distance, int use_max,
                                        int n_threads, int64_t* out_idx,
                                        float* out_val) {
    set_threads(n_threads);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < n_curves; c++) {
        int64_t* idx = out_idx + c * n_peaks;
        float* val = out_val + c * n_peaks;
        int64_t k = orc_find_top_peaks(data + c * flat_len, flat_len, n_peaks,
                                       min_distance, use_max, idx, val);
        for (int64_t i = k; i < n_peaks; i++) {
            idx[i] = -1;
            val[i] = 0.0f;
        }
    }
}
