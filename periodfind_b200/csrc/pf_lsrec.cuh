// pf_lsrec.cuh -- Lomb-Scargle on a uniform frequency grid by an
// angle-addition recurrence along the grid.
//
// Included by the two semantics units after pf_fold.cuh (same namespace).
//
// The chosen LS fold evaluates sin and cos of 2 pi frac(t * f) for every
// (point, frequency): two MUFU operations per evaluation, which bound it.
// When the trial frequencies are f_k = f0 + k * df exactly, consecutive
// phases of one point differ by the same angle d = 2 pi t df, so
//     (cos, sin)(theta_{k+1}) = (c cos d - s sin d, s cos d + c sin d).
// Here a thread owns R consecutive frequencies: per point it takes the
// split-precision phase and one MUFU sin/cos pair at its first frequency,
// then R - 1 rotations (two multiplies and two fused multiply-adds each),
// with four accumulations per frequency as the sincos form.  (cos d, sin d)
// depend on the point only: the CTA computes them once per staged point, in
// FP64 (sincospi of the fraction of t * df), and every thread reuses them.
// Per evaluation that is 2 / R MUFU operations instead of 2.
//
// Error: the first pair carries the MUFU error of the sincos form; each
// rotation adds at most a few f32 roundings (the rotation pair is correctly
// rounded from FP64), so after R - 1 steps the values are within ~R times
// the f32 rounding of the sincos form's.  The autotuner offers R = 4 and 8.
#pragma once

namespace pfk {
namespace PF_KNS {

constexpr uint32_t kRecTile = 512;  // points staged per tile

// One item: curve w.curve, frequencies w.p0 .. w.p0 + w.np - 1 (w.np <=
// BLOCK * R); thread tid owns frequencies w.p0 + tid * R + r, r < R.
template <int BLOCK, int R>
__device__ __forceinline__ void lsrec_item(const FoldParams& p, const WorkItem w, uint32_t item) {
    extern __shared__ __align__(16) unsigned char smem[];
    float4* tile = reinterpret_cast<float4*>(smem);  // (t, y, cos d, sin d)

    stamp_start(p, item);
    const CurveDesc cd = p.curves[w.curve];
    const uint32_t n = cd.n;
    const int tid = threadIdx.x;
    const uint32_t j0 = (uint32_t)tid * R;
    const bool active = j0 < w.np;
    const uint32_t k0 = w.p0 + (active ? j0 : 0u);
    const double f = p.f0 + (double)k0 * p.df;
    Cell s;
    cell_setup_freq(s, f);
    // The split-precision phase needs |t f| < 2^21 over the CTA (as the
    // sincos form): the largest |f| of the item is at one of its ends.
    const double f_last = p.f0 + (double)(w.p0 + w.np - 1u) * p.df;
    const double fmax_cta = fmax(fabs(p.f0 + (double)w.p0 * p.df), fabs(f_last));
    const double tmax = (double)__uint_as_float(*p.tmax_bits);
    const bool alt = !(tmax * fmax_cta < 2097152.0);  // uniform over the CTA

    float acc[R][4];
#pragma unroll
    for (int r = 0; r < R; r++) acc[r][0] = acc[r][1] = acc[r][2] = acc[r][3] = 0.0f;

    for (uint32_t base = 0; base < n; base += kRecTile) {
        const uint32_t cnt = min(kRecTile, n - base);
        __syncthreads();
        for (uint32_t i = tid; i < cnt; i += BLOCK) {
            const float t = p.t[cd.off + base + i];
            const float y = p.m[cd.off + base + i];
            // d = 2 pi frac(t df): the product in FP64 (t df is within a few
            // thousand turns; its rounding is ~1e-13 turns), its fraction in
            // [-0.5, 0.5] turns, then sin / cos of pi * 2 frac.
            const double x = (double)t * p.df;
            const double fr = x - rint(x);
            double sd, cdv;
            sincospi(2.0 * fr, &sd, &cdv);
            tile[i] = make_float4(t, y, (float)cdv, (float)sd);
        }
        __syncthreads();
        if (!active) continue;
#pragma unroll 2
        for (uint32_t i = 0; i < cnt; i++) {
            const float4 pt = tile[i];
            float ph;
            if (alt) ph = fold_exact<false>((double)pt.x, s);
            else ph = fold_df<false>(pt.x, s);
            float sn, cs;
            sincosf(kTwoPi * ph, &sn, &cs);
#pragma unroll
            for (int r = 0; r < R; r++) {
                acc[r][0] = __fmaf_rn(pt.y, cs, acc[r][0]);
                acc[r][1] = __fmaf_rn(pt.y, sn, acc[r][1]);
                acc[r][2] = __fmaf_rn(cs, cs, acc[r][2]);
                acc[r][3] = __fmaf_rn(cs, sn, acc[r][3]);
                if (r + 1 < R) {
                    const float c2 = __fmaf_rn(cs, pt.z, -__fmul_rn(sn, pt.w));
                    sn = __fmaf_rn(sn, pt.z, __fmul_rn(cs, pt.w));
                    cs = c2;
                }
            }
        }
    }
    if (active) {
        float* out = p.out + (size_t)w.curve * p.n_per;
#pragma unroll
        for (int r = 0; r < R; r++) {
            const uint32_t k = k0 + (uint32_t)r;
            if (j0 + (uint32_t)r < w.np) {
                const LSAcc a{acc[r][0], acc[r][1], acc[r][2], acc[r][3]};
                out[k] = ls_power(a, n);
            }
        }
    }
    stamp_end(p, item);
}

// Items from the device work queue (an item is BLOCK * R consecutive
// frequencies), persistently or one CTA per item.  Compiled for 1024
// resident threads per SM at R = 4 (58 registers) and 768 at R = 8 (its 32
// accumulators spill at 64 registers).
template <int BLOCK, int R, bool PERSIST>
__global__ void __launch_bounds__(BLOCK, (R >= 8 ? 3 : 4) * 256 / BLOCK)
    lsrec_kernel(const FoldParams p) {
    if constexpr (PERSIST) {
        for_each_queued_item<BLOCK * R>(p, [&](const WorkItem& w, uint32_t k) {
            lsrec_item<BLOCK, R>(p, w, k);
        });
    } else {
        lsrec_item<BLOCK, R>(p, queue_item<BLOCK * R>(p, blockIdx.x), blockIdx.x);
    }
}

}  // namespace PF_KNS
}  // namespace pfk
