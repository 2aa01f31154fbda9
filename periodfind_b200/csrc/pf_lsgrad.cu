// pf_lsgrad.cu -- Lomb-Scargle power with derivatives at arbitrary angular
// frequencies: forward (power, dP/domega, d2P/domega2 and the least-squares
// coefficients), backward (dP/dy and the frequency gradient) and Newton
// refinement of peaks off the trial grid.  None of this has a counterpart in
// the reference, which evaluates the power on the trial grid only
// (periodfind/cuda/ls.cu:75-136, rust/src/ls.rs:231-276).
//
// The power.  With v = (C, S) = (sum y cos th, sum y sin th) and
// M = [[CC, CS], [CS, SS]] (CC = sum cos^2 th, CS = sum cos th sin th,
// SS = N - CC), the reference's tau-rotated expression
//   P = 0.5 (A^2 / D_l + B^2 / D_r)        (ls.cu:107-129)
// equals 0.5 v^T M^-1 v for every tau, because tau only diagonalises M: P is
// half the squared norm of the least-squares projection of y onto
// (cos th, sin th).  So with w = (alpha, beta) = M^-1 v:
//   P        = 0.5 w . v
//   dP/dy_i  = alpha cos th_i + beta sin th_i
//   dP/dw    = w . v' - 0.5 w^T M' w
//   d2P/dw2  = u^T M^-1 u + w . v'' - 0.5 w^T M'' w,   u = v' - M' w
// where ' is d/domega with th_i = omega (t_i - t0).  P does not depend on t0
// (a time shift rotates (cos, sin) jointly), so t0 is the midpoint of each
// curve's time span, which keeps the t and t^2 weights small.  w does depend
// on t0: every kernel here derives t0 the same way (exact min/max).
//
// Arithmetic: the phase omega dt / 2pi is a split-precision FP32 product of
// float pairs (FP64 for |f dt| >= 2^21 turns), the sine and cosine come from
// the MUFU unit, all sums are FP32, and the closed form above is evaluated
// in FP64 once per (curve, frequency).  Degenerate M (det <= 1e-6 CC SS, e.g. one point or
// all phases equal) gives power 0 and zero derivatives, as the reference's
// zero denominators give 0 (ls.cu:131-134).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "pf_launch.h"

namespace pfk {

namespace {

constexpr int kLsThreads = 256;
constexpr int kLsWarps = kLsThreads / 32;
constexpr uint32_t kLsTile = 2048;        // staged points (16 B each)
constexpr uint32_t kGradFreqTile = 512;   // staged frequencies in the backward
constexpr double kInv2Pi = 0.15915494309189533577;
constexpr double kShift = 6755399441055744.0;  // 1.5 * 2^52
// det(M) / (CC SS) is the squared sine of the angle between the cos and sin
// vectors; below this M is treated as singular (FP32 sums leave rounding
// residue where it is exactly singular, e.g. one point).
constexpr double kDegenerate = 1e-6;
// Newton refinement returns its last iterate unless that iterate's power is
// more than this fraction below the best evaluated one.
constexpr double kKeepLast = 1e-5;

struct Sums {
    float C, S, CC, CS;
    float C1, S1, CC1, CS1;
    float C2, S2, CC2, CS2;
};

// An unevaluated float pair hi + lo.  A time measured from the curve's t0
// (t an f32, t0 the midpoint of two f32 values) has at most 26 significant
// bits, so hi + lo holds it exactly.
struct F2 {
    float hi, lo;
};
__device__ __forceinline__ F2 split2(double v) {
    F2 r;
    r.hi = __double2float_rn(v);
    r.lo = __double2float_rn(v - (double)r.hi);
    return r;
}

// A staged point: its time from t0 as a float pair (dh is also the FP32
// derivative weight) and its magnitude.
struct __align__(16) StagedPoint {
    float dh, dl, y, unused;
};

struct Deriv {
    double P, P1, P2, alpha, beta;
};

// Phase in turns of frequency f (turns per time unit) at time dt, reduced to
// about [-0.5, 0.5].  Split precision (the default): the product of the two
// float pairs as p + e, with p = RN(fh * dh) and e its exact rounding error
// (one fma) plus the cross terms fh * dl + fl * dh (fl * dl is below 2^-40
// of the product); the integer part is removed from p exactly (|p| < 2^22);
// the phase is good to the f32 rounding of the result, as the FP64
// reduction below.  Needs |f dt| < 2^21 (checked by the callers).
__device__ __forceinline__ float phase_df(F2 f, F2 d) {
    const float p = __fmul_rn(f.hi, d.hi);
    float e = __fmaf_rn(f.hi, d.hi, -p);
    e = __fmaf_rn(f.hi, d.lo, e);
    e = __fmaf_rn(f.lo, d.hi, e);
    const float n = __fsub_rn(__fadd_rn(p, 12582912.0f), 12582912.0f);  // rint, |p| < 2^22
    return __fadd_rn(__fsub_rn(p, n), e);
}
// FP64 reduction for frequencies or spans beyond that range.
__device__ __forceinline__ float phase_f64(double f, double dt) {
    const double u = f * dt;
    const double n = __dsub_rn(__dadd_rn(u, kShift), kShift);
    return (float)__dsub_rn(u, n);
}
// sine and cosine of 2 pi * phase (|phase| <= ~0.5): the MUFU unit (absolute
// error ~4e-7, inside every tolerance of these derivatives).
__device__ __forceinline__ void sincos_turns(float ph, float* s, float* c) {
    __sincosf(6.28318530717958647692f * ph, s, c);
}
constexpr double kDfLimit = 2097152.0;  // 2^21 turns

template <int ORDER>
__device__ __forceinline__ void add_point(Sums& a, float x, float y, float s, float c) {
    a.C = fmaf(y, c, a.C);
    a.S = fmaf(y, s, a.S);
    a.CC = fmaf(c, c, a.CC);
    a.CS = fmaf(c, s, a.CS);
    if constexpr (ORDER >= 1) {
        const float yx = y * x;
        const float s2 = 2.0f * s * c;           // sin 2th
        const float c2 = fmaf(c, c, -s * s);     // cos 2th
        a.C1 = fmaf(-yx, s, a.C1);
        a.S1 = fmaf(yx, c, a.S1);
        a.CC1 = fmaf(-x, s2, a.CC1);
        a.CS1 = fmaf(x, c2, a.CS1);
        if constexpr (ORDER >= 2) {
            const float yxx = yx * x, xx2 = 2.0f * x * x;
            a.C2 = fmaf(-yxx, c, a.C2);
            a.S2 = fmaf(-yxx, s, a.S2);
            a.CC2 = fmaf(-xx2, c2, a.CC2);
            a.CS2 = fmaf(-xx2, s2, a.CS2);
        }
    }
}

// XOR butterfly: every lane ends with the same, bit-identical totals.
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

template <int ORDER>
__device__ __forceinline__ void warp_reduce(Sums& a) {
    a.C = warp_sum(a.C);
    a.S = warp_sum(a.S);
    a.CC = warp_sum(a.CC);
    a.CS = warp_sum(a.CS);
    if constexpr (ORDER >= 1) {
        a.C1 = warp_sum(a.C1);
        a.S1 = warp_sum(a.S1);
        a.CC1 = warp_sum(a.CC1);
        a.CS1 = warp_sum(a.CS1);
    }
    if constexpr (ORDER >= 2) {
        a.C2 = warp_sum(a.C2);
        a.S2 = warp_sum(a.S2);
        a.CC2 = warp_sum(a.CC2);
        a.CS2 = warp_sum(a.CS2);
    }
}

template <int ORDER>
__device__ Deriv finish(const Sums& a, uint32_t n) {
    Deriv d{0.0, 0.0, 0.0, 0.0, 0.0};
    const double C = a.C, S = a.S, CC = a.CC, CS = a.CS;
    const double SS = (double)n - CC;
    const double det = CC * SS - CS * CS;
    if (!(det > kDegenerate * CC * SS)) return d;
    const double al = (SS * C - CS * S) / det;
    const double be = (CC * S - CS * C) / det;
    d.alpha = al;
    d.beta = be;
    d.P = 0.5 * (al * C + be * S);
    if constexpr (ORDER >= 1) {
        const double C1 = a.C1, S1 = a.S1, CC1 = a.CC1, CS1 = a.CS1;
        d.P1 = al * C1 + be * S1 - 0.5 * ((al * al - be * be) * CC1 + 2.0 * al * be * CS1);
        if constexpr (ORDER >= 2) {
            const double C2 = a.C2, S2 = a.S2, CC2 = a.CC2, CS2 = a.CS2;
            const double u0 = C1 - (CC1 * al + CS1 * be);
            const double u1 = S1 - (CS1 * al - CC1 * be);
            const double quad = (SS * u0 * u0 - 2.0 * CS * u0 * u1 + CC * u1 * u1) / det;
            d.P2 = quad + al * C2 + be * S2 -
                   0.5 * ((al * al - be * be) * CC2 + 2.0 * al * be * CS2);
        }
    }
    return d;
}

// Midpoint of the curve's time span (exact min / max, so every kernel and
// every CTA derives the same t0) and the half span.  Block-wide; all threads
// must call it.
__device__ double curve_t0(const float* __restrict__ t, int64_t o, uint32_t n,
                           double* half_span) {
    __shared__ float red_lo[kLsWarps], red_hi[kLsWarps];
    float lo = INFINITY, hi = -INFINITY;
    for (uint32_t i = threadIdx.x; i < n; i += kLsThreads) {
        const float v = t[o + i];
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
    }
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) {
        lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, k));
        hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, k));
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();  // red_* may still be read from an earlier call
    if (lane == 0) {
        red_lo[wid] = lo;
        red_hi[wid] = hi;
    }
    __syncthreads();
    lo = red_lo[0];
    hi = red_hi[0];
#pragma unroll
    for (int w = 1; w < kLsWarps; w++) {
        lo = fminf(lo, red_lo[w]);
        hi = fmaxf(hi, red_hi[w]);
    }
    *half_span = n ? 0.5 * ((double)hi - (double)lo) : 0.0;
    return n ? 0.5 * ((double)lo + (double)hi) : 0.0;
}

// One CTA per (curve, group of kLsWarps * rounds frequencies); a warp per
// frequency, lanes striding over the staged points, sums reduced by warp
// shuffles.  REFINE runs the safeguarded Newton iteration for each
// frequency inside the kernel (n_steps updates, n_steps + 1 evaluations).
// Newton steps where d2P/domega2 < 0, otherwise a quarter-bracket step
// uphill; every iterate is clamped to [omega0 - h, omega0 + h].
template <int ORDER, bool REFINE>
__global__ void __launch_bounds__(kLsThreads)
    ls_eval_kernel(LsEvalParams p, uint32_t rounds, uint32_t groups) {
    __shared__ StagedPoint tile[kLsTile];
    const uint64_t c = blockIdx.x / groups;
    const uint32_t g = blockIdx.x % groups;
    const int64_t o = p.off[c];
    const uint32_t n = (uint32_t)(p.off[c + 1] - o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double half_span;
    const double t0 = curve_t0(p.t, o, n, &half_span);
    const uint32_t ntiles = (n + kLsTile - 1) / kLsTile;
    const uint32_t n_eval = REFINE ? p.n_steps + 1 : 1;

    for (uint32_t j = 0; j < rounds; j++) {
        const uint64_t k = (uint64_t)g * kLsWarps * rounds + (uint64_t)j * kLsWarps + wid;
        const bool valid = k < p.n_freq;
        const uint64_t cell = c * p.n_freq + k;
        double w = valid ? p.omega[c * p.omega_stride + k] : 0.0;
        double hw = 0.0, lo_b = 0.0, hi_b = 0.0, best_w = w, best_P = -1.0;
        double last_w = w, last_P = -1.0;
        if (REFINE && valid) {
            hw = p.half_width[cell];
            lo_b = w - hw;
            hi_b = w + hw;
        }
        for (uint32_t e = 0; e < n_eval; e++) {
            const double f = w * kInv2Pi;
            const F2 fp = split2(f);
            const bool df = fabs(f) * half_span < kDfLimit;  // uniform per warp
            Sums a{};
            for (uint32_t tt = 0; tt < ntiles; tt++) {
                const uint32_t base = tt * kLsTile;
                const uint32_t cnt = min(kLsTile, n - base);
                if (ntiles > 1 || (j == 0 && e == 0)) {
                    __syncthreads();
                    for (uint32_t i = threadIdx.x; i < cnt; i += kLsThreads) {
                        const F2 d = split2((double)p.t[o + base + i] - t0);
                        tile[i] = StagedPoint{d.hi, d.lo, p.y[o + base + i], 0.0f};
                    }
                    __syncthreads();
                }
                if (df) {
                    for (uint32_t i = lane; i < cnt; i += 32) {
                        const StagedPoint q = tile[i];
                        float s, cs;
                        sincos_turns(phase_df(fp, F2{q.dh, q.dl}), &s, &cs);
                        add_point<ORDER>(a, q.dh, q.y, s, cs);
                    }
                } else {
                    for (uint32_t i = lane; i < cnt; i += 32) {
                        const StagedPoint q = tile[i];
                        float s, cs;
                        sincos_turns(phase_f64(f, (double)q.dh + (double)q.dl), &s, &cs);
                        add_point<ORDER>(a, q.dh, q.y, s, cs);
                    }
                }
            }
            warp_reduce<ORDER>(a);
            const Deriv d = finish<ORDER>(a, n);
            if constexpr (REFINE) {
                last_P = d.P;
                last_w = w;
                if (d.P > best_P) {
                    best_P = d.P;
                    best_w = w;
                }
                if (e + 1 < n_eval) {
                    // Newton toward the maximum; where the curvature does not
                    // point to one, a quarter-bracket step uphill.
                    double step = (d.P2 < 0.0) ? -d.P1 / d.P2
                                               : ((d.P1 > 0.0) ? 0.25 * hw : -0.25 * hw);
                    w = fmin(fmax(w + step, lo_b), hi_b);
                }
            } else if (valid && lane == 0) {
                p.power[cell] = (float)d.P;
                if (p.dpdw) p.dpdw[cell] = (float)d.P1;
                if (p.d2pdw2) p.d2pdw2[cell] = (float)d.P2;
                if (p.coef) {
                    p.coef[2 * cell] = (float)d.alpha;
                    p.coef[2 * cell + 1] = (float)d.beta;
                }
            }
        }
        if (REFINE && valid && lane == 0) {
            // The last iterate unless it fell clearly below the best one:
            // near a converged maximum the powers of the iterates differ by
            // rounding only, and picking the largest would pick by noise.
            const bool keep_last = last_P >= best_P * (1.0 - kKeepLast);
            p.omega_out[cell] = keep_last ? last_w : best_w;
            p.power[cell] = (float)fmax(keep_last ? last_P : best_P, 0.0);
        }
    }
}

// dP/dy: a thread per point, summing g_k (alpha_k cos th_ik + beta_k sin
// th_ik) over the curve's frequencies staged in shared memory; CTAs of point
// tile 0 also write the frequency gradient g_k * dP/domega_k.
__global__ void __launch_bounds__(kLsThreads)
    ls_grad_kernel(LsGradParams p) {
    __shared__ double sf[kGradFreqTile];
    __shared__ float sfh[kGradFreqTile], sfl[kGradFreqTile];
    __shared__ float sa[kGradFreqTile], sb[kGradFreqTile];
    const uint64_t c = blockIdx.y;
    const int64_t o = p.off[c];
    const uint32_t n = (uint32_t)(p.off[c + 1] - o);
    const uint32_t i = blockIdx.x * kLsThreads + threadIdx.x;
    const bool head = blockIdx.x == 0;
    if (!head && blockIdx.x * kLsThreads >= n) return;  // whole CTA past the curve
    double half_span;
    const double t0 = curve_t0(p.t, o, n, &half_span);
    const bool have = i < n;
    const double dt = have ? (double)p.t[o + i] - t0 : 0.0;
    const F2 d = split2(dt);
    float acc = 0.0f;
    for (uint64_t k0 = 0; k0 < p.n_freq; k0 += kGradFreqTile) {
        const uint32_t cnt = (uint32_t)min((uint64_t)kGradFreqTile, p.n_freq - k0);
        __syncthreads();
        bool ok = true;
        for (uint32_t q = threadIdx.x; q < cnt; q += kLsThreads) {
            const uint64_t cell = c * p.n_freq + k0 + q;
            const float gp = p.grad_power[cell];
            const double f = p.omega[c * p.omega_stride + k0 + q] * kInv2Pi;
            const F2 fp = split2(f);
            sf[q] = f;
            sfh[q] = fp.hi;
            sfl[q] = fp.lo;
            ok = ok && fabs(f) * half_span < kDfLimit;
            sa[q] = gp * p.coef[2 * cell];
            sb[q] = gp * p.coef[2 * cell + 1];
            if (head && p.grad_omega) p.grad_omega[cell] = (double)(gp * p.dpdw[cell]);
        }
        // Every frequency of the tile within the split-precision range?
        const bool df = __syncthreads_and(ok ? 1 : 0) != 0;
        if (p.grad_mags && have) {
            if (df) {
                for (uint32_t q = 0; q < cnt; q++) {
                    float s, cs;
                    sincos_turns(phase_df(F2{sfh[q], sfl[q]}, d), &s, &cs);
                    acc = fmaf(sa[q], cs, acc);
                    acc = fmaf(sb[q], s, acc);
                }
            } else {
                for (uint32_t q = 0; q < cnt; q++) {
                    float s, cs;
                    sincos_turns(phase_f64(sf[q], dt), &s, &cs);
                    acc = fmaf(sa[q], cs, acc);
                    acc = fmaf(sb[q], s, acc);
                }
            }
        }
    }
    if (p.grad_mags && have) p.grad_mags[o + i] = acc;
}

}  // namespace

static uint32_t eval_rounds(uint64_t n_freq) {
    const uint64_t r = (n_freq + kLsWarps - 1) / kLsWarps;
    return (uint32_t)(r < 8 ? (r ? r : 1) : 8);
}

cudaError_t launch_ls_eval(const LsEvalParams& p, int order, cudaStream_t s) {
    if (p.n_curves == 0 || p.n_freq == 0) return cudaSuccess;
    const uint32_t rounds = eval_rounds(p.n_freq);
    const uint64_t per = (uint64_t)kLsWarps * rounds;
    const uint64_t groups = (p.n_freq + per - 1) / per;
    const uint64_t blocks = p.n_curves * groups;
    if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    if (order <= 0)
        ls_eval_kernel<0, false><<<(unsigned)blocks, kLsThreads, 0, s>>>(p, rounds, (uint32_t)groups);
    else if (order == 1)
        ls_eval_kernel<1, false><<<(unsigned)blocks, kLsThreads, 0, s>>>(p, rounds, (uint32_t)groups);
    else
        ls_eval_kernel<2, false><<<(unsigned)blocks, kLsThreads, 0, s>>>(p, rounds, (uint32_t)groups);
    return cudaGetLastError();
}

cudaError_t launch_ls_refine(const LsEvalParams& p, cudaStream_t s) {
    if (p.n_curves == 0 || p.n_freq == 0) return cudaSuccess;
    const uint32_t rounds = eval_rounds(p.n_freq);
    const uint64_t per = (uint64_t)kLsWarps * rounds;
    const uint64_t groups = (p.n_freq + per - 1) / per;
    const uint64_t blocks = p.n_curves * groups;
    if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    ls_eval_kernel<2, true><<<(unsigned)blocks, kLsThreads, 0, s>>>(p, rounds, (uint32_t)groups);
    return cudaGetLastError();
}

cudaError_t launch_ls_grad(const LsGradParams& p, uint32_t max_len, cudaStream_t s) {
    if (p.n_curves == 0 || p.n_freq == 0) return cudaSuccess;
    if (p.n_curves > 65535) {
        // gridDim.y limit: split the curves into batches.
        for (uint64_t c0 = 0; c0 < p.n_curves; c0 += 65535) {
            LsGradParams q = p;
            q.n_curves = p.n_curves - c0 < 65535 ? p.n_curves - c0 : 65535;
            q.off = p.off + c0;
            q.omega = p.omega + c0 * p.omega_stride;
            q.grad_power += c0 * p.n_freq;
            q.coef += 2 * c0 * p.n_freq;
            q.dpdw += c0 * p.n_freq;
            if (q.grad_omega) q.grad_omega += c0 * p.n_freq;
            cudaError_t e = launch_ls_grad(q, max_len, s);
            if (e != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    const uint32_t tiles =
        (p.grad_mags && max_len) ? (max_len + kLsThreads - 1) / kLsThreads : 1;
    dim3 grid(tiles, (unsigned)p.n_curves);
    ls_grad_kernel<<<grid, kLsThreads, 0, s>>>(p);
    return cudaGetLastError();
}

}  // namespace pfk
