// pf_fold.cuh -- fused fold / bin / statistic kernels for CE, AOV and LS.
//
// Included by exactly two translation units that differ only in compiler
// flags, which is how the reference's two implementations differ:
//   kern_cudasem.cu  -use_fast_math: approximate f32 divides, fast log/sincos,
//                    FTZ, multiply-add contraction -- the reference's CUDA
//                    build (setup.py:129, periodfind/cuda/*.cu).
//   kern_cpusem.cu   IEEE divides, accurate log/sin/cos, no contraction --
//                    the reference's CPU path (rust/src/{fold,ce,aov,ls}.rs).
// Expressions that the reference writes the same way in both are written
// here once, verbatim in shape, so each translation unit reproduces its
// reference's rounding.  Arithmetic that must not depend on the flags
// (the exact fold, fixed-point statistics) uses explicit _rn intrinsics.
//
// Decomposition (thread per cell): a CTA takes one curve, one period
// derivative and up to BLOCK consecutive trial periods; thread j owns trial
// period p0 + j for the whole curve.  The curve is streamed through shared
// memory in tiles of kTile points; every thread of a warp reads the same
// point (a broadcast), so point data costs one shared load per warp-step.
// Each thread's histogram is private and laid out [bin][thread] in shared
// memory, so every warp-wide update hits 32 distinct banks; updates are
// fire-and-forget shared atomics (no read-after-write chain between points).
// The statistic is finished in the same kernel from the private histogram:
// no histogram round trip through global memory (periodfind/cuda/ce.cu:
// 160-167 writes one 4*n_bins-byte histogram per (period, pdt) to HBM).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "pf_launch.h"
#include "pf_types.h"

#ifndef PF_SEM_CPU_TU
#error "define PF_SEM_CPU_TU to 0 (reference CUDA arithmetic) or 1 (reference CPU arithmetic)"
#endif
#ifndef PF_KNS
#error "define PF_KNS, the namespace that keeps this unit's kernels distinct"
#endif

namespace pfk {
// Each including unit gets its own namespace: the two units compile the same
// templates with different arithmetic, so their symbols must not merge.
namespace PF_KNS {

// periodfind/cuda/ls.cu:18 and rust/src/ls.rs:13 (both 6.2831855f).
constexpr float kTwoPi = 6.283185307179586f;

struct Cell {
    float period, pdt_corr;
    double Pd, yhi, ylo, c;
    float fhi, flo, ghi, glo;
};

template <int FOLD>
__device__ __forceinline__ void cell_setup(Cell& s, float period, float period_dt) {
    s.period = period;
    // periodfind/cuda/ce.cu:125, aov.cu:68, ls.cu:65; rust/src/fold.rs:13-15.
    s.pdt_corr = (period_dt / period) / 2;
    if (FOLD == FOLD_EXACT || FOLD == FOLD_DF) {
        // 1/P as a double-double (yhi + ylo): yhi = RN(1/P); the residual
        // 1 - P*yhi is exact in one fma, and ylo = residual * yhi.
        s.Pd = (double)period;
        s.yhi = __drcp_rn(s.Pd);
        const double r = __fma_rn(-s.Pd, s.yhi, 1.0);
        s.ylo = __dmul_rn(r, s.yhi);
        s.c = (double)s.pdt_corr;
    }
    if (FOLD == FOLD_DF) {
        // f = 1/P and g = pdt_corr / P as unevaluated float pairs.
        s.fhi = __double2float_rn(s.yhi);
        s.flo = __double2float_rn(__dadd_rn(__dadd_rn(s.yhi, -(double)s.fhi), s.ylo));
        const double g = __dmul_rn(s.c, s.yhi);
        s.ghi = __double2float_rn(g);
        s.glo = __double2float_rn(__dadd_rn(g, -(double)s.ghi));
    }
}

// A trial frequency f (FP64, exact) instead of a period: 1/P is f itself, so
// the exact fold's double-double reciprocal is (f, 0) and the split-precision
// fold's float pair is f rounded plus its remainder.  No period derivative.
__device__ __forceinline__ void cell_setup_freq(Cell& s, double f) {
    s.period = (float)(1.0 / f);
    s.pdt_corr = 0.0f;
    s.Pd = 1.0 / f;
    s.yhi = f;
    s.ylo = 0.0;
    s.c = 0.0;
    s.fhi = __double2float_rn(f);
    s.flo = __double2float_rn(__dadd_rn(f, -(double)s.fhi));
    s.ghi = s.glo = 0.0f;
}

// The reference fold, operation for operation (periodfind/cuda/ce.cu:140-143,
// aov.cu:106-109, ls.cu:95-97; rust/src/fold.rs:22-26).
__device__ __forceinline__ float fold_ref(float t, const Cell& s) {
    double t_corr_d = (double)t - (double)s.pdt_corr * (double)t * (double)t;
    double ratio_d = t_corr_d / (double)s.period;
    return fabsf((float)(ratio_d - floor(ratio_d)));
}

// Same result as fold_ref without a divide.  For a double a and a period P
// that is an f32 value, the exact quotient a/P is at least 2^-77 (relative)
// away from every rounding midpoint of double precision (a - m*P is a
// nonzero multiple of 2^(e_a - 77) for any 54-bit midpoint m), while
// qh + lo below approximates a/P to ~2^-103.  RN(qh + lo) is therefore the
// correctly rounded quotient, i.e. exactly what the FP64 divide returns.
template <bool HAS_PDT>
__device__ __forceinline__ float fold_exact(double td, const Cell& s) {
    double a;
    if constexpr (HAS_PDT) {
        // Same expression as the reference, so the same contraction.
        a = td - s.c * td * td;
    } else {
        a = td;
    }
    const double qh = __dmul_rn(a, s.yhi);
    const double e = __fma_rn(a, s.yhi, -qh);
    const double lo = __fma_rn(a, s.ylo, e);
    const double q = __dadd_rn(qh, lo);
    return fabsf((float)(q - floor(q)));
}

// All-FP32 fold (precision study only: loses ~1e-3 cycles at 1e4-1e5 cycles).
__device__ __forceinline__ float fold_f32(float t, const Cell& s) {
    const float tc = t - s.pdt_corr * t * t;
    const float r = tc / s.period;
    return fabsf(r - floorf(r));
}

// Split-precision FP32 phase of t_corr / P = t*f - t^2*g (f = 1/P,
// g = pdt_corr / P as float pairs).  Each product is carried as a rounded
// float plus its exact rounding error (fma), the integer part is removed
// from the rounded float (exact for |x| < 2^22, checked per CTA), and the
// small terms are added last.  Before the final rounding the phase is good
// to ~1e-10 turns at 6e4 cycles of baseline; the f32 result is then within
// half an ulp of it (at most 2^-25 turns), the same bound as the reference's
// FP64 fold rounded to f32.  Result in turns, within [-1, 1].
__device__ __forceinline__ float rint_small(float x) {
    return __fsub_rn(__fadd_rn(x, 12582912.0f), 12582912.0f);  // |x| < 2^22
}

// The same phase without a period derivative in four operations: r, the
// integer nearest t*fhi (the exact product against 1.5*2^23 in one FMA: ulp 1
// there, |t*fhi| < 2^22), then t*fhi - r and t*flo each added on the exact
// product in one FMA.  Two roundings of the reduced phase: |error| <= 2^-24
// turns (fold_df: 2^-25 in seven operations).  Used for curves of at least
// kPhase4MinPoints points; on shorter ones the LS sums can be near-singular
// (a two-point curve's power moved by a quarter under a one-ulp phase
// change), and they keep fold_df.
constexpr uint32_t kPhase4MinPoints = 32;
__device__ __forceinline__ float fold_df4(float t, const Cell& s) {
    const float r = __fsub_rn(__fmaf_rn(t, s.fhi, 12582912.0f), 12582912.0f);
    return __fmaf_rn(t, s.flo, __fmaf_rn(t, s.fhi, -r));
}

template <bool HAS_PDT>
__device__ __forceinline__ float fold_df(float t, const Cell& s) {
    const float p = __fmul_rn(t, s.fhi);
    float e = __fmaf_rn(t, s.fhi, -p);
    e = __fmaf_rn(t, s.flo, e);
    float ph = __fsub_rn(p, rint_small(p));
    if constexpr (HAS_PDT) {
        const float t2 = __fmul_rn(t, t);
        const float t2e = __fmaf_rn(t, t, -t2);
        const float p2 = __fmul_rn(t2, s.ghi);
        float e2 = __fmaf_rn(t2, s.ghi, -p2);
        e2 = __fmaf_rn(t2, s.glo, e2);
        e2 = __fmaf_rn(t2e, s.ghi, e2);
        ph = __fsub_rn(ph, __fsub_rn(p2, rint_small(p2)));
        e = __fsub_rn(e, e2);
    }
    return __fadd_rn(ph, e);
}

// Bound on |t_corr / P| over this CTA's cells: max|t| / min|P| +
// |pdt| max|t|^2 / (2 min|P|^2), min|P| over every thread's `my_min_abs_p`.
// All threads of the CTA must call it.
template <int BLOCK>
__device__ double cta_qbound_of(const FoldParams& p, double my_min_abs_p, float period_dt) {
    __shared__ double warp_min[BLOCK / 32];
    double mn = my_min_abs_p;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    if ((threadIdx.x & 31) == 0) warp_min[threadIdx.x >> 5] = mn;
    __syncthreads();
    double pmin = warp_min[0];
#pragma unroll
    for (int k = 1; k < BLOCK / 32; k++) pmin = fmin(pmin, warp_min[k]);
    const double tmax = (double)__uint_as_float(*p.tmax_bits);
    return tmax / pmin + fabs((double)period_dt) * tmax * tmax / (2.0 * pmin * pmin);
}

template <int BLOCK>
__device__ double cta_qbound(const FoldParams& p, uint32_t pi, float period_dt) {
    // On a frequency grid 1 / |f| stands for |P| (f = 0 gives an infinite
    // bound, so the exact fold, whose phase is then 0).
    const double absp = p.fgrid ? 1.0 / fabs(p.f0 + (double)pi * p.df) : fabs((double)p.periods[pi]);
    return cta_qbound_of<BLOCK>(p, absp, period_dt);
}

// Optional per-work-item timing (%globaltimer, ns): the CTA's first thread
// stamps the start; every thread raises the end stamp when it finishes.
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void stamp_start(const FoldParams& p, uint32_t item) {
    if (p.stamps && threadIdx.x == 0) p.stamps[2 * (size_t)item] = global_ns();
}
__device__ __forceinline__ void stamp_end(const FoldParams& p, uint32_t item) {
    if (p.stamps) atomicMax(&p.stamps[2 * (size_t)item + 1], global_ns());
}

// Work item k of the device queue (see WorkQueue).
template <int BLOCK>
__device__ __forceinline__ WorkItem queue_item(const FoldParams& p, uint32_t k) {
    const uint32_t tiles = (p.n_per + BLOCK - 1) / BLOCK;
    const uint32_t tpc = tiles * p.n_pdt;
    const uint32_t ci = k / tpc, rem = k - ci * tpc;
    const uint32_t d = rem / tiles, tile = rem - d * tiles;
    WorkItem w;
    w.curve = p.q.order[ci];
    w.pdt = d;
    w.p0 = tile * BLOCK;
    w.np = min((uint32_t)BLOCK, p.n_per - w.p0);
    return w;
}

// Persistent CTA loop: take the next item from the queue until it is empty.
// The leading barrier keeps the previous item's shared memory (tile,
// counters, the item slot) in use until every thread has finished with it.
// (Claiming the next item during the current one was measured: no gain, and
// a register spill in the LS fold.)
template <int BLOCK, class F>
__device__ __forceinline__ void for_each_queued_item(const FoldParams& p, F&& f) {
    __shared__ uint32_t s_item;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) s_item = atomicAdd(p.q.next, 1u);
        __syncthreads();
        const uint32_t k = s_item;
        if (k >= p.q.n_work) break;
        f(queue_item<BLOCK>(p, k), k);
    }
}

// Resident CTAs per SM the queue kernels are compiled for (registers held
// so that occupancy is not lost to the register allocator; measured): the LS
// folds and the AOV bin kernel at 5 x 256 threads, the CE bin kernel at its
// shared-memory limit of 4 x 256 (CE 10 x 10).
template <int ALGO, int BLOCK>
constexpr int queue_min_blocks() {
    return (ALGO == ALGO_CE ? 4 : 5) * 256 / BLOCK;
}

// trunc(q) for finite q in [0, 2^23): identical to the reference's
// (size_t) conversion on that range, without a conversion instruction.
__device__ __forceinline__ unsigned trunc_u(float q) {
    return __float_as_uint(__fadd_rz(q, 8388608.0f)) - 0x4B000000u;
}

template <int FOLD>
using tile_t_type = typename std::conditional<FOLD == FOLD_EXACT, double, float>::type;

// Private per-thread accumulators (LS) and shared-memory views of one CTA.
struct Views {
    float* tile_tf;
    double* tile_td;
    uint32_t* tile_a;
    unsigned long long* tile_a64;
    uint32_t* hist;               // CE counts, [slot][BLOCK]
    unsigned long long* hist64;   // AOV FIX, [slot][BLOCK]
    uint32_t* a_cnt;              // AOV F32, [bin][BLOCK] x 3
    float* a_sum;
    float* a_sq;
};

struct LSAcc {
    float mag_cos, mag_sin, cos_cos, cos_sin;
};

// The LS power from a cell's sums (periodfind/cuda/ls.cu:144-165 /
// rust/src/ls.rs:253-280), n points.
__device__ __forceinline__ float ls_power(const LSAcc& ls, uint32_t n) {
    const float mag_cos = ls.mag_cos, mag_sin = ls.mag_sin;
    const float cos_cos = ls.cos_cos, cos_sin = ls.cos_sin;
    float sin_sin = static_cast<float>(n) - cos_cos;
    float cos_tau, sin_tau;
    sincosf(0.5f * atan2f(2.0f * cos_sin, cos_cos - sin_sin), &sin_tau, &cos_tau);
    float numerator_l = cos_tau * mag_cos + sin_tau * mag_sin;
    numerator_l *= numerator_l;
    float numerator_r = cos_tau * mag_sin - sin_tau * mag_cos;
    numerator_r *= numerator_r;
    float denominator_l = cos_tau * cos_tau * cos_cos + 2 * cos_tau * sin_tau * cos_sin +
                          sin_tau * sin_tau * sin_sin;
    float denominator_r = cos_tau * cos_tau * sin_sin - 2 * cos_tau * sin_tau * cos_sin +
                          sin_tau * sin_tau * cos_cos;
#if PF_SEM_CPU_TU
    return (denominator_l == 0.0f || denominator_r == 0.0f)
               ? 0.0f
               : 0.5f * (numerator_l / denominator_l + numerator_r / denominator_r);
#else
    return 0.5f * ((numerator_l / denominator_l) + (numerator_r / denominator_r));
#endif
}

// Stream the curve through shared memory and accumulate this thread's cell.
template <int ALGO, int FOLD, int ACC, int BLOCK, bool OVL, bool HAS_PDT, bool ALT>
__device__ __forceinline__ void accumulate(const FoldParams& p, const Views& v, const Cell& s,
                                           int64_t off, uint32_t n, bool active, LSAcc& ls) {
    using TT = tile_t_type<FOLD>;
    TT* tile_t;
    if constexpr (FOLD == FOLD_EXACT) tile_t = v.tile_td; else tile_t = v.tile_tf;
    const int tid = threadIdx.x;
    const uint32_t nP = p.n_phase, nM = p.n_mag;
    const uint32_t po = p.p_overlap, mo = p.m_overlap;
    const float phase_bin_size = p.phase_bin_size;

    for (uint32_t base = 0; base < n; base += kTile) {
        const uint32_t cnt = min(kTile, n - base);
        __syncthreads();
        // Stage the tile with 16-byte loads (curves start 16-byte aligned
        // and are padded to a multiple of 4 points).
        {
            const float4* gt = reinterpret_cast<const float4*>(p.t + off + base);
            const uint32_t n4 = (cnt + 3) >> 2;
            for (uint32_t i4 = tid; i4 < n4; i4 += BLOCK) {
                const float4 q = gt[i4];
                tile_t[4 * i4 + 0] = (TT)q.x;
                tile_t[4 * i4 + 1] = (TT)q.y;
                tile_t[4 * i4 + 2] = (TT)q.z;
                tile_t[4 * i4 + 3] = (TT)q.w;
            }
            if constexpr (ALGO == ALGO_CE) {
                const uint4* ga = reinterpret_cast<const uint4*>(p.aux32 + off + base);
                uint4* sa = reinterpret_cast<uint4*>(v.tile_a);
                for (uint32_t i4 = tid; i4 < n4; i4 += BLOCK) sa[i4] = ga[i4];
            } else if constexpr (ALGO == ALGO_AOV && ACC == AOVACC_FIX) {
                const ulonglong2* ga = reinterpret_cast<const ulonglong2*>(p.aux64 + off + base);
                ulonglong2* sa = reinterpret_cast<ulonglong2*>(v.tile_a64);
                for (uint32_t i2 = tid; i2 < 2 * n4; i2 += BLOCK) sa[i2] = ga[i2];
            } else {
                const uint4* ga = reinterpret_cast<const uint4*>(p.m + off + base);
                uint4* sa = reinterpret_cast<uint4*>(v.tile_a);
                for (uint32_t i4 = tid; i4 < n4; i4 += BLOCK) sa[i4] = ga[i4];
            }
        }
        __syncthreads();
        if (!active) continue;

        if constexpr (ALGO == ALGO_LS && FOLD == FOLD_DF && !ALT) {
            // Four points per pair of 128-bit broadcast loads; the tail (not
            // the zero padding) one point at a time.  The phase form is
            // uniform over the CTA (one curve per item).
            auto ls_tile = [&](auto phase_of) {
                auto ls_point = [&](float t, float mag) {
                    const float ph = phase_of(t);
                    float sin_val, cos_val;
                    sincosf(kTwoPi * ph, &sin_val, &cos_val);
                    ls.mag_cos += mag * cos_val;
                    ls.mag_sin += mag * sin_val;
                    ls.cos_cos += cos_val * cos_val;
                    ls.cos_sin += cos_val * sin_val;
                };
                const float4* t4 = reinterpret_cast<const float4*>(tile_t);
                const float4* m4 = reinterpret_cast<const float4*>(v.tile_a);
                const uint32_t full = cnt & ~3u;
#pragma unroll 2
                for (uint32_t i = 0; i < full; i += 4) {
                    const float4 tt = t4[i >> 2], mm = m4[i >> 2];
                    ls_point(tt.x, mm.x);
                    ls_point(tt.y, mm.y);
                    ls_point(tt.z, mm.z);
                    ls_point(tt.w, mm.w);
                }
                for (uint32_t i = full; i < cnt; i++)
                    ls_point(tile_t[i], __uint_as_float(v.tile_a[i]));
            };
            if (!HAS_PDT && n >= kPhase4MinPoints)
                ls_tile([&](float t) { return fold_df4(t, s); });
            else
                ls_tile([&](float t) { return fold_df<HAS_PDT>(t, s); });
            continue;
        }

#pragma unroll 4
        for (uint32_t i = 0; i < cnt; i++) {
            float folded;
            if constexpr (FOLD == FOLD_REF) {
                folded = fold_ref(tile_t[i], s);
            } else if constexpr (FOLD == FOLD_EXACT) {
                folded = fold_exact<HAS_PDT>(tile_t[i], s);
            } else if constexpr (FOLD == FOLD_F32) {
                folded = fold_f32(tile_t[i], s);
            } else if constexpr (ALT) {
                // Outside the split-precision range: the exact fold.
                folded = fold_exact<HAS_PDT>((double)tile_t[i], s);
            } else {
                folded = fold_df<HAS_PDT>(tile_t[i], s);
            }

            if constexpr (ALGO == ALGO_LS) {
                // periodfind/cuda/ls.cu:92-104; rust/src/ls.rs:242-251.
                const float mag = __uint_as_float(v.tile_a[i]);
                float sin_val, cos_val;
                sincosf(kTwoPi * folded, &sin_val, &cos_val);
                ls.mag_cos += mag * cos_val;
                ls.mag_sin += mag * sin_val;
                ls.cos_cos += cos_val * cos_val;
                ls.cos_sin += cos_val * sin_val;
            } else {
                // PhaseBin: (size_t)(folded / phase_bin_size)  (ce.cu:66-68,
                // aov.cu:35-37; ce.rs:78, aov.rs:172).  folded <= 1, so the
                // bin is at most n_phase (the reference wraps it with %).
                const unsigned pb = min(trunc_u(folded / phase_bin_size), nP);
                if constexpr (ALGO == ALGO_CE) {
                    const uint32_t a = v.tile_a[i];
                    if constexpr (!OVL) {
                        // Row n_phase is folded into row 0 after the loop.
                        atomicAdd(&v.hist[(pb * nM + a) * BLOCK + tid], 1u);
                    } else {
                        // ce.cu:148-155 / ce.rs:82-89 with wrapping bins.
                        const uint32_t mb = a & 0x7FFFFFFFu;
                        const bool sat = (a >> 31) != 0u;
                        for (uint32_t ii = 0; ii < po; ii++) {
                            const uint32_t row = (pb + ii) % nP;
                            for (uint32_t jj = 0; jj < mo; jj++) {
                                const uint32_t col =
                                    sat ? (jj == 0 ? mb : (jj - 1) % nM) : (mb + jj) % nM;
                                atomicAdd(&v.hist[(row * nM + col) * BLOCK + tid], 1u);
                            }
                        }
                    }
                } else {  // AOV
                    if constexpr (ACC == AOVACC_FIX) {
                        const unsigned long long q = v.tile_a64[i];
                        if constexpr (!OVL) {
                            atomicAdd(&v.hist64[pb * BLOCK + tid], q);
                        } else {
                            for (uint32_t o = 0; o < po; o++)
                                atomicAdd(&v.hist64[((pb + o) % nP) * BLOCK + tid], q);
                        }
                    } else {
                        // aov.cu:111-122 / aov.rs:173-180, in point order.
                        const float mag = __uint_as_float(v.tile_a[i]);
                        const float mag_sq = mag * mag;
                        if constexpr (!OVL) {
                            const uint32_t b = (pb >= nP) ? pb - nP : pb;
                            atomicAdd(&v.a_cnt[b * BLOCK + tid], 1u);
                            atomicAdd(&v.a_sum[b * BLOCK + tid], mag);
                            atomicAdd(&v.a_sq[b * BLOCK + tid], mag_sq);
                        } else {
                            for (uint32_t o = 0; o < po; o++) {
                                const uint32_t b = (pb + o) % nP;
                                atomicAdd(&v.a_cnt[b * BLOCK + tid], 1u);
                                atomicAdd(&v.a_sum[b * BLOCK + tid], mag);
                                atomicAdd(&v.a_sq[b * BLOCK + tid], mag_sq);
                            }
                        }
                    }
                }
            }
        }
    }
}

template <int ALGO, int FOLD, int ACC, int BLOCK, bool OVL>
__device__ __forceinline__ void fold_item(const FoldParams& p, const WorkItem w, uint32_t item) {
    using TT = tile_t_type<FOLD>;
    extern __shared__ __align__(16) unsigned char smem[];
    constexpr size_t kAuxBytes = (ALGO == ALGO_AOV && ACC == AOVACC_FIX) ? 8 : 4;
    unsigned char* after_t = smem + kTile * sizeof(TT);
    unsigned char* hist_raw = after_t + kTile * kAuxBytes;

    const uint32_t nP = p.n_phase, nM = p.n_mag;
    const uint32_t po = p.p_overlap, mo = p.m_overlap;

    Views v;
    v.tile_tf = reinterpret_cast<float*>(smem);
    v.tile_td = reinterpret_cast<double*>(smem);
    v.tile_a = reinterpret_cast<uint32_t*>(after_t);
    v.tile_a64 = reinterpret_cast<unsigned long long*>(after_t);
    v.hist = reinterpret_cast<uint32_t*>(hist_raw);
    v.hist64 = reinterpret_cast<unsigned long long*>(hist_raw);
    v.a_cnt = reinterpret_cast<uint32_t*>(hist_raw);
    v.a_sum = reinterpret_cast<float*>(hist_raw) + (size_t)nP * BLOCK;
    v.a_sq = reinterpret_cast<float*>(hist_raw) + (size_t)2 * nP * BLOCK;

    stamp_start(p, item);
    const CurveDesc cd = p.curves[w.curve];
    const uint32_t n = cd.n;
    const int tid = threadIdx.x;
    const bool active = (uint32_t)tid < w.np;
    const uint32_t pi = w.p0 + (active ? (uint32_t)tid : 0u);
    const float period_dt = p.pdts[w.pdt];

    Cell s;
    if (ALGO == ALGO_LS && p.fgrid) cell_setup_freq(s, p.f0 + (double)pi * p.df);
    else cell_setup<FOLD>(s, p.periods[pi], period_dt);

    // Zero this thread's column of the private histogram.
    if constexpr (ALGO == ALGO_CE) {
        const uint32_t slots = (OVL ? nP : nP + 1) * nM;
        for (uint32_t k = 0; k < slots; k++) v.hist[k * BLOCK + tid] = 0u;
    } else if constexpr (ALGO == ALGO_AOV) {
        if constexpr (ACC == AOVACC_FIX) {
            const uint32_t slots = OVL ? nP : nP + 1;
            for (uint32_t k = 0; k < slots; k++) v.hist64[k * BLOCK + tid] = 0ull;
        } else {
            for (uint32_t k = 0; k < nP; k++) {
                v.a_cnt[k * BLOCK + tid] = 0u;
                v.a_sum[k * BLOCK + tid] = 0.0f;
                v.a_sq[k * BLOCK + tid] = 0.0f;
            }
        }
    }

    LSAcc ls{0.0f, 0.0f, 0.0f, 0.0f};
    // The split-precision fold needs |t_corr / P| < 2^21 (uniform per CTA).
    bool alt = false;
    if constexpr (FOLD == FOLD_DF) alt = !(cta_qbound<BLOCK>(p, pi, period_dt) < 2097152.0);
    // The period derivative is uniform over the CTA: pick the loop once.
    if (period_dt != 0.0f) {
        if (alt) accumulate<ALGO, FOLD, ACC, BLOCK, OVL, true, true>(p, v, s, cd.off, n, active, ls);
        else accumulate<ALGO, FOLD, ACC, BLOCK, OVL, true, false>(p, v, s, cd.off, n, active, ls);
    } else {
        if (alt) accumulate<ALGO, FOLD, ACC, BLOCK, OVL, false, true>(p, v, s, cd.off, n, active, ls);
        else accumulate<ALGO, FOLD, ACC, BLOCK, OVL, false, false>(p, v, s, cd.off, n, active, ls);
    }

    if (!active) {
        stamp_end(p, item);
        return;
    }
    const size_t out_idx =
        (size_t)w.curve * ((size_t)p.n_per * p.n_pdt) + (size_t)pi * p.n_pdt + w.pdt;

    if constexpr (ALGO == ALGO_CE) {
        uint32_t* hist = v.hist;
        if constexpr (!OVL) {
            for (uint32_t mb = 0; mb < nM; mb++)
                hist[mb * BLOCK + tid] += hist[(nP * nM + mb) * BLOCK + tid];
        }
        if (p.bins) {
            uint32_t* o = p.bins + out_idx * ((size_t)nP * nM);
            for (uint32_t k = 0; k < nP * nM; k++) o[k] = hist[k * BLOCK + tid];
        }
        const float divf = (float)((unsigned long long)n * po * mo);
        float ce = 0.0f;
        for (uint32_t j = 0; j < nP; j++) {
            float p_j = 0.0f;
            for (uint32_t i = 0; i < nM; i++) p_j += (float)hist[(j * nM + i) * BLOCK + tid] / divf;
#if PF_SEM_CPU_TU
            // rust/src/ce.rs:96-110: one running sum over all cells.
            for (uint32_t i = 0; i < nM; i++) {
                const float p_ij = (float)hist[(j * nM + i) * BLOCK + tid] / divf;
                if (p_ij != 0.0f) ce += p_ij * logf(p_j / p_ij);
            }
#else
            // periodfind/cuda/ce.cu:231-243: per-phase-row contribution,
            // then the rows are summed (here in row order).
            float ce_contrib = 0.0f;
            for (uint32_t i = 0; i < nM; i++) {
                const float p_ij = (float)hist[(j * nM + i) * BLOCK + tid] / divf;
                if (p_ij != 0) ce_contrib += p_ij * logf(p_j / p_ij);
            }
            ce += ce_contrib;
#endif
        }
        p.out[out_idx] = ce;
    } else if constexpr (ALGO == ALGO_AOV) {
        if constexpr (ACC == AOVACC_FIX) {
            unsigned long long* hist64 = v.hist64;
            if constexpr (!OVL) hist64[tid] += hist64[nP * BLOCK + tid];
            if (p.bins) {
                uint32_t* o = p.bins + out_idx * (size_t)nP;
                for (uint32_t b = 0; b < nP; b++)
                    o[b] = (uint32_t)(hist64[b * BLOCK + tid] >> kFixCountShift);
            }
            const unsigned long long mask = (1ull << kFixCountShift) - 1ull;
            const double xbar = cd.fix_sumx / (double)n;
            double s1 = 0.0, sbx = 0.0;
            for (uint32_t b = 0; b < nP; b++) {
                const unsigned long long h = hist64[b * BLOCK + tid];
                const unsigned long long c = h >> kFixCountShift;
                if (c != 0ull) {
                    const double nb = (double)c;
                    const double X = (double)(h & mask);
                    const double mu = X / nb;
                    const double r = mu - xbar;
                    s1 = __fma_rn(nb * r, r, s1);
                    sbx = __fma_rn(X, mu, sbx);
                }
            }
            const double s2 = __dadd_rn((double)po * cd.fix_sumx2, -sbx);
            const double scale = ((double)n - (double)nP) / ((double)nP - 1.0);
            float res;
#if PF_SEM_CPU_TU
            res = (s2 <= 0.0) ? 0.0f : (float)(scale * (s1 / s2));  // aov.rs:197-201
#else
            res = (float)(scale * (s1 / (s2 <= 0.0 ? 0.0 : s2)));      // aov.cu:242-244
#endif
            p.out[out_idx] = res;
        } else {
            // periodfind/cuda/aov.cu:225-244 / rust/src/aov.rs:184-201.
            if (p.bins) {
                uint32_t* o = p.bins + out_idx * (size_t)nP;
                for (uint32_t b = 0; b < nP; b++) o[b] = v.a_cnt[b * BLOCK + tid];
            }
            const float avg = cd.avg;
            float s1 = 0;
            float s2 = 0;
            for (uint32_t b = 0; b < nP; b++) {
                float nn = static_cast<float>(v.a_cnt[b * BLOCK + tid]);
                float sum = v.a_sum[b * BLOCK + tid];
                float sq_sum = v.a_sq[b * BLOCK + tid];
                if (nn != 0) {
                    float aux = sum / nn;
                    float residual = aux - avg;
                    s1 += nn * residual * residual;
                    s2 += sq_sum - nn * aux * aux;
                }
            }
            const float length = (float)n;
#if PF_SEM_CPU_TU
            p.out[out_idx] = (s2 == 0.0f)
                                 ? 0.0f
                                 : ((length - (float)nP) / ((float)nP - 1.0f)) * (s1 / s2);
#else
            p.out[out_idx] = (static_cast<float>(length - nP) / static_cast<float>(nP - 1)) *
                             (s1 / s2);
#endif
        }
    } else {
        p.out[out_idx] = ls_power(ls, n);
    }
    stamp_end(p, item);
}

// The chosen folds (exact, split-precision) take items from the device
// queue, persistently (PERSIST) or one CTA per item; the reference fold and
// the all-FP32 study fold take one CTA per item of the host-built list, as
// the reference launches.
template <int ALGO, int FOLD, int ACC, int BLOCK, bool OVL, bool PERSIST>
__global__ void __launch_bounds__(BLOCK, (ALGO == ALGO_LS && uses_queue(KIND_FOLD, FOLD))
                                             ? queue_min_blocks<ALGO_LS, BLOCK>()
                                             : 1)
    fold_kernel(const FoldParams p) {
    if constexpr (!uses_queue(KIND_FOLD, FOLD)) {
        fold_item<ALGO, FOLD, ACC, BLOCK, OVL>(p, p.work[blockIdx.x], blockIdx.x);
    } else if constexpr (PERSIST) {
        for_each_queued_item<BLOCK>(p, [&](const WorkItem& w, uint32_t k) {
            fold_item<ALGO, FOLD, ACC, BLOCK, OVL>(p, w, k);
        });
    } else {
        fold_item<ALGO, FOLD, ACC, BLOCK, OVL>(p, queue_item<BLOCK>(p, blockIdx.x), blockIdx.x);
    }
}

// ------------------------------------------------------------- preparation

// CE magnitude bins, once per point (the reference recomputes
// MagBin(mags[idx]) for every (point, period), ce.cu:146).  Stored as
// (mag_bin % n_mag) | (saturated << 31); a saturated bin is 2^64-1, whose
// wrapped successors are 0, 1, ... (size_t arithmetic, ce.cu:150-152).
__global__ void ce_magbin_kernel(const float* __restrict__ m, uint32_t* __restrict__ aux,
                                 const CurveDesc* __restrict__ curves, uint32_t n_curves,
                                 uint32_t n_mag, float mag_bin_size, int flag_saturated) {
    const uint32_t c = blockIdx.x;
    if (c >= n_curves) return;
    const CurveDesc cd = curves[c];
    const uint32_t n4 = (cd.n + 3u) & ~3u;
    for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x) {
        uint32_t v = 0;
        if (i < cd.n) {
            const float mag_val = m[cd.off + i];
            const unsigned long long mb = static_cast<unsigned long long>(mag_val / mag_bin_size);
            v = (uint32_t)(mb % n_mag);
            if (flag_saturated && mb == ~0ull) v |= 0x80000000u;
        }
        aux[cd.off + i] = v;
    }
}

// Folded phase of each (period, time) pair with one fold variant, as the
// fold kernels compute it (precision studies): out[p * n + i].  FOLD_DF
// returns turns in [-1, 1] (the four-operation form where the LS kernel uses
// it: no derivative and n >= kPhase4MinPoints); the others [0, 1].
template <int FOLD>
__global__ void phase_probe_kernel(const float* __restrict__ t, uint64_t n,
                                   const float* __restrict__ periods, uint64_t n_per,
                                   float period_dt, float* __restrict__ out) {
    const uint64_t total = n * n_per;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t pi = k / n, i = k % n;
        Cell s;
        cell_setup<FOLD>(s, periods[pi], period_dt);
        const float ti = t[i];
        float ph;
        if constexpr (FOLD == FOLD_REF) {
            ph = fold_ref(ti, s);
        } else if constexpr (FOLD == FOLD_EXACT) {
            ph = (period_dt != 0.0f) ? fold_exact<true>((double)ti, s)
                                     : fold_exact<false>((double)ti, s);
        } else if constexpr (FOLD == FOLD_F32) {
            ph = fold_f32(ti, s);
        } else {
            ph = (period_dt != 0.0f) ? fold_df<true>(ti, s)
                 : (n >= kPhase4MinPoints) ? fold_df4(ti, s)
                                           : fold_df<false>(ti, s);
        }
        out[k] = ph;
    }
}

}  // namespace PF_KNS
}  // namespace pfk
