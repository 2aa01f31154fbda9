// pf_bin.cuh -- the chosen form's fused fold+bin kernel for CE and AOV.
//
// Included by the two semantics units after pf_fold.cuh (same namespace).
//
// Per (point, trial period) the reference computes
//     q = RN(t_corr / P)                  (FP64 divide)
//     folded = (float)(q - floor(q))      (FP64 floor, f64->f32 convert)
//     bin = (size_t)(folded / bin_size)   (f32 divide)
// which on B200 puts three instructions per evaluation on the narrow XU
// pipe (floor, conversion, the divide's reciprocal), ~16 ops/clk/SM.
// Here the bin comes from three FP64 operations and integer arithmetic:
//     q' = t_corr * RN(1/P)               within 2 ulp of RN(t_corr / P)
//     r  = RD(q' + 1.5*2^52)              low word = floor(q')
//     y  = RD(q' * n*2^20 + 1.5*2^52)     mantissa = 2^51 + floor(q'*n*2^20)
//     row = (y >> 20) - n*floor(q')       = floor(frac(q') * n)  (mod 2^32)
// The 20 low bits of y are frac(q')*n's fractional bits.  The reference's
// quotient folded / bin_size differs from frac(q')*n by less than a bound
// delta(n) (f32 divide, bin-width rounding, f64->f32 rounding of the phase,
// and q' versus RN(t_corr/P); computed on the host).  When frac(q')*n lies
// within that bound of an integer the evaluation recomputes the reference's
// exact sequence (the correctly rounded quotient via fold_exact, then the
// float fold and divide), so bin occupancies are identical by construction;
// about 3e-5 of evaluations take that branch at n = 10.
//
// Valid while |q| * n < 2^30 (checked per CTA from the batch's max|t|;
// otherwise the CTA runs the generic loop).  While also |q| < 2^19 one FP64
// operation does it (fast_bin32): y = RD(t_corr * (RN(1/P) * 2^32) +
// 1.5*2^52) on the exact product leaves floor(frac(q') * 2^32) in its low
// word f, and the 64-bit product f * n holds the row (high word) and the
// position within it (low word, tested against the same guard in units of
// 2^-32, widened by n + 2 for the truncation).
//
// CE counters are 16-bit halves of 32-bit words when every count fits
// (curve length * overlaps < 65536), doubling the CTAs per SM; AOV keeps a
// 32-bit count and a 32-bit fixed-point magnitude sum per bin.  Updates are
// `red.shared.add.u32` (no return value, no dependency chain).
#pragma once

namespace pfk {
namespace PF_KNS {

// Fire-and-forget shared reduction.  No "memory" clobber: the counters it
// updates are never read inside the point loop, so the compiler may hoist
// the next points' shared loads above it (independent point chains overlap).
// The epilogue's counter reads are ordered after the loop by an explicit
// compiler barrier plus __syncwarp().
__device__ __forceinline__ void red_shared_u32(uint32_t addr, uint32_t v) {
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(addr), "r"(v));
}

__device__ __forceinline__ void compiler_fence() { asm volatile("" ::: "memory"); }

__device__ __forceinline__ uint32_t lds_u32(uint32_t addr) {
    uint32_t v;
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}

constexpr double kMagic15 = 6755399441055744.0;  // 1.5 * 2^52

// One CTA: curve w.curve, period derivative w.pdt, periods p0 .. p0+np-1
// (one per thread).  Shared memory: [tile of 16-byte point records
// {double t; u32 a; u32 b}][counters].  CE: a = byte offset of the
// magnitude column within a phase row, b = increment (1 or 1 << 16).
// AOV: a = fixed-point magnitude.
struct BinPoint {
    double t;
    uint32_t a, b;
};

// c log2 c of a count (zero for c = 0 and 1): one log per bin, no divide,
// ln 2 applied once at the end.  A count (< 2^16 here: the bin kernels run
// curves of fewer than 65536 points) becomes a float exactly by placing it
// in the mantissa of 2^23, which costs a bitwise OR and an add instead of an
// integer-to-float conversion.  Explicit roundings, so that every kernel
// that sums these terms in the same order gets the same bits.
__device__ __forceinline__ float ce_xlx(uint32_t c) {
    const float f = __fsub_rn(__uint_as_float(c | 0x4B000000u), 8388608.0f);
    return __fmul_rn(f, log2f(fmaxf(f, 1.0f)));
}

// CE of one cell from its running sum of row terms, over n points.
__device__ __forceinline__ float ce_finish(float acc, uint32_t n) {
    return __fmul_rn(acc, 0.69314718055994531f / (float)n);
}

// AOV of one cell from sum_b X_b^2 / c_b (fixed-point bin sums X_b).
__device__ __forceinline__ float aov_finish(double sbx, const CurveDesc& cd, uint32_t n,
                                            uint32_t nP) {
    const double s1 = fmax(sbx - cd.fix_sumx * cd.fix_sumx / (double)n, 0.0);
    const double s2 = __dadd_rn(cd.fix_sumx2, -sbx);
    const double scale = ((double)n - (double)nP) / ((double)nP - 1.0);
#if PF_SEM_CPU_TU
    return (s2 <= 0.0) ? 0.0f : (float)(scale * (s1 / s2));
#else
    return (float)(scale * (s1 / (s2 <= 0.0 ? 0.0 : s2)));
#endif
}

// The chosen form's CE statistic.  Counters are read through 32-bit shared
// addresses (tbase = this thread's column).  Each row term
// C_j ln C_j - sum_i c_ij ln c_ij is non-negative, so FP32 accumulation keeps
// the relative error near 1e-7 (FP64 here costs registers in the binning
// loop, measured slower).  Per row, the magnitude bins are taken in pairs
// (the two 16-bit halves of a word).
template <bool CNT16>
__device__ __forceinline__ float ce_stat_fast(uint32_t tbase, uint32_t nP, uint32_t W,
                                              uint32_t block, uint32_t n) {
    auto xlx = [](uint32_t c) -> float { return ce_xlx(c); };
    float acc = 0.0f;
    for (uint32_t j = 0; j < nP; j++) {
        uint32_t col = 0;
        float row = 0.0f;
        for (uint32_t wi = 0; wi < W; wi++) {
            const uint32_t wv = lds_u32(tbase + (j * W + wi) * block * 4u);
            if constexpr (CNT16) {
                // Both 16-bit halves summed at once: each half's column
                // total is at most n < 2^16, so no carry crosses halves.
                col += wv;
                row = __fadd_rn(row, __fadd_rn(xlx(wv & 0xFFFFu), xlx(wv >> 16)));
            } else {
                col += wv;
                row = __fadd_rn(row, xlx(wv));
            }
        }
        if constexpr (CNT16) col = (col & 0xFFFFu) + (col >> 16);
        acc = __fadd_rn(acc, __fsub_rn(xlx(col), row));
    }
    return ce_finish(acc, n);
}

// The chosen form's AOV sum_b X_b^2 / c_b over the fixed-point bin sums X_b
// (empty bins have X_b = 0 and contribute nothing).  Counters [bin][count,
// sum][thread].
__device__ __forceinline__ double aov_sbx_fast(uint32_t tbase, uint32_t nP, uint32_t block) {
    double sbx = 0.0;
    for (uint32_t b = 0; b < nP; b++) {
        const uint32_t c = lds_u32(tbase + 2u * b * block * 4u);
        const double Xd = (double)lds_u32(tbase + (2u * b + 1u) * block * 4u);
        sbx = __fma_rn(__dmul_rn(Xd, Xd), __drcp_rn((double)max(c, 1u)), sbx);
    }
    return sbx;
}

// Statistic forms.  REF_STATS: the reference's operation sequence
// (periodfind/cuda/ce.cu:160-178, aov.cu:84-121), so identical bins give
// values bit-identical to the plain form.  Otherwise the same statistic
// computed from the integer bins with one log (CE) or one reciprocal (AOV)
// per bin and no divide:
//   CE  = (sum_j C_j ln C_j - sum_ij c_ij ln c_ij) / n,  C_j = sum_i c_ij
//         (the bin counts c over n points; the reference's p_ij ln(p_j/p_ij)
//         summed, with the 1/n scale taken out of the logs);
//   AOV = (n - nP)/(nP - 1) * s1 / s2, s1 = sum_b X_b^2 / c_b - X^2 / n,
//         s2 = sum x^2 - sum_b X_b^2 / c_b (X_b the fixed-point bin sums).
template <int ALGO, bool CNT16, int BLOCK, bool REF_STATS, int ROUNDS>
__device__ __forceinline__ void bin_item(const FoldParams& p, const WorkItem w, uint32_t item) {
    extern __shared__ __align__(16) unsigned char smem[];
    // CE: one 16-byte record per point.  AOV: the times (doubles) and the
    // fixed-point magnitudes in two arrays, so four points take three
    // 128-bit loads instead of four.
    BinPoint* tile = reinterpret_cast<BinPoint*>(smem);
    double* tile_t = reinterpret_cast<double*>(smem);
    uint32_t* tile_a = reinterpret_cast<uint32_t*>(smem + kBinTile * sizeof(double));
    unsigned char* cnt_raw = smem + kBinTile * sizeof(BinPoint);
    const uint32_t cnt_base = (uint32_t)__cvta_generic_to_shared(cnt_raw);

    stamp_start(p, item);
    const CurveDesc cd = p.curves[w.curve];
    const uint32_t n = cd.n;
    const int tid = threadIdx.x;
    const float period_dt = p.pdts[w.pdt];
    const uint32_t nP = p.n_phase, nM = p.n_mag;

    // Counter layout: CE  [nP rows][W words][BLOCK] u32, W = nM or ceil(nM/2)
    //                 AOV [nP][2][BLOCK] u32 (count, fixed-point sum): a bin's
    //                 sum lies a constant BLOCK words after its count, so the
    //                 second reduction takes an immediate address offset.
    const uint32_t W = (ALGO == ALGO_CE) ? (CNT16 ? (nM + 1) / 2 : nM) : 1;
    const uint32_t row_stride = W * BLOCK * 4;  // bytes per phase row
    const uint32_t slots = (ALGO == ALGO_CE) ? nP * W : 2 * nP;
    const uint32_t tbase = cnt_base + tid * 4;

    // The item covers ROUNDS x BLOCK periods; thread tid takes period
    // p0 + r * BLOCK + tid in round r.  Range guard for y = q * n * 2^20 over
    // every round (uniform over the CTA).  The cell constants (1 / P as a
    // double-double, pdt / 2P) are finite exactly when P is finite and non-zero
    // and pdt is finite; non-finite periods or derivatives (device-pointer
    // callers are not checked on the host) take the generic loop, whose bins
    // are always clamped.
    bool fin = isfinite(period_dt);
    double my_pmin = INFINITY;
#pragma unroll
    for (int r = 0; r < ROUNDS; r++) {
        const uint32_t j = (uint32_t)(r * BLOCK + tid);
        const float per = p.periods[w.p0 + (j < w.np ? j : 0u)];
        fin = fin && isfinite(per) && per != 0.0f;
        my_pmin = fmin(my_pmin, fabs((double)per));
    }
    const double qb = cta_qbound_of<BLOCK>(p, my_pmin, period_dt);
    const bool fast = __syncthreads_and(fin ? 1 : 0) && qb * (double)nP < 1073741824.0;  // 2^30
    // |q| < 2^19 as well: the phase's 32 fraction bits come from one FMA.
    const bool fast32 = fast && qb < 524288.0;

    const double nd20 = (double)nP * 1048576.0;
    const uint32_t n_neg = 0u - nP;
    // Edge test: ((ylo + D) mod 2^20) < 2D, as one IMAD and one compare on
    // the fraction bits moved to the top of the word.
    const uint32_t edge_add = p.edge_d << 12;
    const uint32_t edge_lim = (2u * p.edge_d) << 12;
    // The same guard in units of 2^-32 of a bin for fast_bin32, widened by
    // n_phase + 2 units for the truncation of the phase to 32 bits.
    const uint32_t edge32_add = edge_add + nP + 2u;
    const uint32_t edge32_lim = 2u * edge32_add;

    auto stage = [&](uint32_t base, uint32_t cnt) {
        const float4* gt = reinterpret_cast<const float4*>(p.t + cd.off + base);
        const uint32_t n4 = (cnt + 3) >> 2;
        if constexpr (ALGO == ALGO_CE) {
            const uint4* ga = reinterpret_cast<const uint4*>(p.aux64 + cd.off + base);
            for (uint32_t i4 = tid; i4 < n4; i4 += BLOCK) {
                const float4 q = gt[i4];
                const uint4 a01 = ga[2 * i4], a23 = ga[2 * i4 + 1];
                // Counter word within a phase row -> byte offset for this
                // CTA shape (the prepared data does not depend on BLOCK).
                constexpr uint32_t kColBytes = BLOCK * 4u;
                tile[4 * i4 + 0] = BinPoint{(double)q.x, a01.x * kColBytes, a01.y};
                tile[4 * i4 + 1] = BinPoint{(double)q.y, a01.z * kColBytes, a01.w};
                tile[4 * i4 + 2] = BinPoint{(double)q.z, a23.x * kColBytes, a23.y};
                tile[4 * i4 + 3] = BinPoint{(double)q.w, a23.z * kColBytes, a23.w};
            }
        } else {
            const uint4* ga = reinterpret_cast<const uint4*>(p.aux32 + cd.off + base);
            for (uint32_t i4 = tid; i4 < n4; i4 += BLOCK) {
                const float4 q = gt[i4];
                const uint4 a = ga[i4];
                reinterpret_cast<double2*>(tile_t)[2 * i4] = make_double2(q.x, q.y);
                reinterpret_cast<double2*>(tile_t)[2 * i4 + 1] = make_double2(q.z, q.w);
                reinterpret_cast<uint4*>(tile_a)[i4] = a;
            }
        }
    };
    // A curve that fits one tile is staged once for every round.
    const bool one_tile = n <= kBinTile;
    if (one_tile) {
        __syncthreads();
        stage(0, n);
        __syncthreads();
    }

#pragma unroll 1
    for (int r = 0; r < ROUNDS; r++) {
    const uint32_t jr = (uint32_t)(r * BLOCK + tid);
    const bool active = jr < w.np;
    const uint32_t pi = w.p0 + (active ? jr : 0u);
    Cell s;
    cell_setup<FOLD_EXACT>(s, p.periods[pi], period_dt);
    const double y32 = s.yhi * 4294967296.0;  // RN(1/P) * 2^32, exact
    for (uint32_t k = 0; k < slots; k++)
        reinterpret_cast<uint32_t*>(cnt_raw)[k * BLOCK + tid] = 0u;

    for (uint32_t base = 0; base < n; base += kBinTile) {
        const uint32_t cnt = min(kBinTile, n - base);
        if (!one_tile) {
            __syncthreads();
            stage(base, cnt);
            __syncthreads();
        }
        if (!active) continue;

        // One point: a 128-bit shared load of its record (CE), or its time
        // and magnitude from the two arrays (AOV).
        auto load_point = [&](uint32_t i) -> BinPoint {
            if constexpr (ALGO == ALGO_CE) {
                const uint4 raw = reinterpret_cast<const uint4*>(tile)[i];
                return BinPoint{__hiloint2double((int)raw.y, (int)raw.x), raw.z, raw.w};
            } else {
                return BinPoint{tile_t[i], tile_a[i], 0u};
            }
        };
        // Fast bin of one point: row (+2^31 bias) and the edge-test value
        // ((fraction + D) << 12); the point is near an edge iff ev < edge_lim.
        auto fast_bin = [&](double td, auto has_pdt_tag, uint32_t& ev) -> uint32_t {
            constexpr bool HAS_PDT = decltype(has_pdt_tag)::value;
            double a;
            if constexpr (HAS_PDT) {
                a = td - s.c * td * td;
            } else {
                a = td;
            }
            const double qh = __dmul_rn(a, s.yhi);
            const double r = __dadd_rd(qh, kMagic15);
            const double y = __fma_rd(qh, nd20, kMagic15);
            const uint32_t ylo = (uint32_t)__double2loint(y);
            const uint32_t yhi = (uint32_t)__double2hiint(y);
            ev = ylo * 4096u + edge_add;
            return __funnelshift_r(ylo, yhi, 20) + (uint32_t)__double2loint(r) * n_neg;
        };
        // |q| < 2^19: y = RD(t_corr * (RN(1/P) * 2^32) + 1.5*2^52), one FMA
        // on the exact product (closer to t_corr / P than the rounded
        // product fast_bin uses, so the same guard holds), leaves
        // floor(frac(q') * 2^32) in its low word f.  The 64-bit product
        // f * n then holds the row in its high word and the position within
        // the row in its low word (plus the guard, for the edge test): one
        // FP64 operation and one integer multiply per point.  The row
        // carries no bias.
        auto fast_bin32 = [&](double td, auto has_pdt_tag, uint32_t& ev) -> uint32_t {
            constexpr bool HAS_PDT = decltype(has_pdt_tag)::value;
            double a;
            if constexpr (HAS_PDT) {
                a = td - s.c * td * td;
            } else {
                a = td;
            }
            const double y = __fma_rd(a, y32, kMagic15);
            const uint32_t f = (uint32_t)__double2loint(y);
            const unsigned long long fn = (unsigned long long)f * nP;
            ev = (uint32_t)fn + edge32_add;
            return (uint32_t)(fn >> 32);
        };
        // The reference's exact sequence (correctly rounded quotient, float
        // fold, f32 divide, then % n_phase: a folded phase of 1.0f gives bin
        // n_phase, which wraps to 0): the bin (+2^31 bias).
        auto exact_bin = [&](double td, auto has_pdt_tag) -> uint32_t {
            constexpr bool HAS_PDT = decltype(has_pdt_tag)::value;
            const float folded = fold_exact<HAS_PDT>(td, s);
            const uint32_t pb = min(trunc_u(folded / p.phase_bin_size), nP);
            return 0x80000000u + (pb == nP ? 0u : pb);
        };
        // AOV bytes per bin row, kept opaque to the compiler so that the
        // counter address is one multiply-add (a power-of-two constant
        // would become a shift and a separate add).
        uint32_t aov_row_bytes = 2 * BLOCK * 4;
        asm("" : "+r"(aov_row_bytes));
        auto add = [&](uint32_t row, const BinPoint& pt, uint32_t sign) {
            // sign is 1 (add) or 0xFFFFFFFF (take back); u32 wraparound keeps
            // packed 16-bit halves and sums exact.
            if constexpr (ALGO == ALGO_CE) {
                red_shared_u32(row * row_stride + pt.a + tbase, pt.b * sign);
            } else {
                const uint32_t a0 = row * aov_row_bytes + tbase;
                red_shared_u32(a0, sign);
                red_shared_u32(a0 + BLOCK * 4, pt.a * sign);
            }
        };

        auto body = [&](auto has_pdt_tag, auto fast_tag, auto f32_tag) {
            constexpr bool FAST = decltype(fast_tag)::value;
            constexpr bool F32 = decltype(f32_tag)::value;
            // Fast bin (unbiased with F32, +2^31 otherwise; the counter
            // address is the same either way) and its edge limit.
            auto bin_of = [&](double td, uint32_t& ev) -> uint32_t {
                if constexpr (F32) return fast_bin32(td, has_pdt_tag, ev);
                else return fast_bin(td, has_pdt_tag, ev);
            };
            const uint32_t lim = F32 ? edge32_lim : edge_lim;
            if constexpr (FAST) {
                // Groups of 32 points: no branch per point; a group whose
                // smallest edge-test value is below the limit is revisited
                // and its near-edge points are moved to the reference's bin.
                for (uint32_t g = 0; g < cnt; g += 32) {
                    const uint32_t gend = min(g + 32u, cnt);
                    uint32_t emin = 0xFFFFFFFFu;
                    if (gend - g == 32u) {
                        // A full group unrolled completely: no loop control
                        // per point (measured 10% faster than unrolling by 4).
                        // Two running minima of the edge test (even and
                        // odd points), so the minimum is two short
                        // dependency chains instead of one of 32 links.
                        uint32_t emin_b = 0xFFFFFFFFu;
                        auto one = [&](const BinPoint& pt, uint32_t& em) {
                            uint32_t ev;
                            const uint32_t row = bin_of(pt.t, ev);
                            em = min(em, ev);
                            add(row, pt, 1u);
                        };
                        if constexpr (ALGO == ALGO_CE) {
#pragma unroll
                            for (uint32_t ii = 0; ii < 32u; ii += 2) {
                                one(load_point(g + ii), emin);
                                one(load_point(g + ii + 1), emin_b);
                            }
                        } else {
                            // Four points per two 128-bit loads of times
                            // and one of magnitudes (g is a multiple of 32).
                            const double2* t2 = reinterpret_cast<const double2*>(tile_t) + g / 2;
                            const uint4* a4 = reinterpret_cast<const uint4*>(tile_a) + g / 4;
#pragma unroll 4
                            for (uint32_t ii = 0; ii < 8u; ii++) {
                                const double2 ta = t2[2 * ii], tb = t2[2 * ii + 1];
                                const uint4 aa = a4[ii];
                                one(BinPoint{ta.x, aa.x, 0u}, emin);
                                one(BinPoint{ta.y, aa.y, 0u}, emin_b);
                                one(BinPoint{tb.x, aa.z, 0u}, emin);
                                one(BinPoint{tb.y, aa.w, 0u}, emin_b);
                            }
                        }
                        emin = min(emin, emin_b);
                    } else {
#pragma unroll 4
                        for (uint32_t i = g; i < gend; i++) {
                            const BinPoint pt = load_point(i);
                            uint32_t ev;
                            const uint32_t row = bin_of(pt.t, ev);
                            emin = min(emin, ev);
                            add(row, pt, 1u);
                        }
                    }
                    if (emin < lim) {
                        for (uint32_t i = g; i < gend; i++) {
                            const BinPoint pt = load_point(i);
                            uint32_t ev;
                            const uint32_t row = bin_of(pt.t, ev);
                            if (ev < lim) {
                                const uint32_t ex =
                                    exact_bin(pt.t, has_pdt_tag) - (F32 ? 0x80000000u : 0u);
                                if (ex != row) {
                                    add(row, pt, 0xFFFFFFFFu);
                                    add(ex, pt, 1u);
                                }
                            }
                        }
                    }
                }
            } else {
#pragma unroll 4
                for (uint32_t i = 0; i < cnt; i++) {
                    const BinPoint pt = load_point(i);
                    add(exact_bin(pt.t, has_pdt_tag), pt, 1u);
                }
            }
        };
        using T_ = std::true_type;
        using F_ = std::false_type;
        if (period_dt != 0.0f) {
            if (fast32) body(T_{}, T_{}, T_{});
            else if (fast) body(T_{}, T_{}, F_{});
            else body(T_{}, F_{}, F_{});
        } else {
            if (fast32) body(F_{}, T_{}, T_{});
            else if (fast) body(F_{}, T_{}, F_{});
            else body(F_{}, F_{}, F_{});
        }
    }
    // Every lane of the warp reaches this barrier (inactive lanes skip the
    // statistic after it).
    compiler_fence();
    __syncwarp();
    if (active) {
    const size_t out_idx =
        (size_t)w.curve * ((size_t)p.n_per * p.n_pdt) + (size_t)pi * p.n_pdt + w.pdt;
    uint32_t* cnt32 = reinterpret_cast<uint32_t*>(cnt_raw);

    if constexpr (ALGO == ALGO_CE && !REF_STATS) {
        p.out[out_idx] = ce_stat_fast<CNT16>(tbase, nP, W, BLOCK, n);
    } else if constexpr (ALGO == ALGO_AOV && !REF_STATS) {
        p.out[out_idx] = aov_finish(aov_sbx_fast(tbase, nP, BLOCK), cd, n, nP);
    } else if constexpr (ALGO == ALGO_CE) {
        auto count = [&](uint32_t j, uint32_t i) -> uint32_t {
            if constexpr (CNT16) {
                const uint32_t wv = cnt32[(j * W + (i >> 1)) * BLOCK + tid];
                return (i & 1u) ? (wv >> 16) : (wv & 0xFFFFu);
            } else {
                return cnt32[(j * W + i) * BLOCK + tid];
            }
        };
        if (p.bins) {
            uint32_t* o = p.bins + out_idx * ((size_t)nP * nM);
            for (uint32_t j = 0; j < nP; j++)
                for (uint32_t i = 0; i < nM; i++) o[j * nM + i] = count(j, i);
        }
        const float divf = (float)((unsigned long long)n * p.p_overlap * p.m_overlap);
        float ce = 0.0f;
        for (uint32_t j = 0; j < nP; j++) {
            float p_j = 0.0f;
            for (uint32_t i = 0; i < nM; i++) p_j += (float)count(j, i) / divf;
#if PF_SEM_CPU_TU
            for (uint32_t i = 0; i < nM; i++) {
                const float p_ij = (float)count(j, i) / divf;
                if (p_ij != 0.0f) ce += p_ij * logf(p_j / p_ij);
            }
#else
            float ce_contrib = 0.0f;
            for (uint32_t i = 0; i < nM; i++) {
                const float p_ij = (float)count(j, i) / divf;
                if (p_ij != 0) ce_contrib += p_ij * logf(p_j / p_ij);
            }
            ce += ce_contrib;
#endif
        }
        p.out[out_idx] = ce;
    } else {
        const uint32_t* sums = cnt32 + BLOCK;
        if (p.bins) {
            uint32_t* o = p.bins + out_idx * (size_t)nP;
            for (uint32_t b = 0; b < nP; b++) o[b] = cnt32[2 * b * BLOCK + tid];
        }
        const double xbar = cd.fix_sumx / (double)n;
        double s1 = 0.0, sbx = 0.0;
        for (uint32_t b = 0; b < nP; b++) {
            const uint32_t c = cnt32[2 * b * BLOCK + tid];
            const uint32_t X = sums[2 * b * BLOCK + tid];
            if (c != 0u) {
                const double nb = (double)c;
                const double Xd = (double)X;
                const double mu = Xd / nb;
                const double r = mu - xbar;
                s1 = __fma_rn(nb * r, r, s1);
                sbx = __fma_rn(Xd, mu, sbx);
            }
        }
        const double s2 = __dadd_rn(cd.fix_sumx2, -sbx);
        const double scale = ((double)n - (double)nP) / ((double)nP - 1.0);
#if PF_SEM_CPU_TU
        p.out[out_idx] = (s2 <= 0.0) ? 0.0f : (float)(scale * (s1 / s2));
#else
        p.out[out_idx] = (float)(scale * (s1 / (s2 <= 0.0 ? 0.0 : s2)));
#endif
    }
    }  // active
    }  // rounds
    stamp_end(p, item);
}

// Items from the device work queue (see WorkQueue), persistently or one CTA
// per item; an item is ROUNDS x BLOCK consecutive periods.
template <int ALGO, bool CNT16, int BLOCK, bool REF_STATS, bool PERSIST, int ROUNDS>
__global__ void __launch_bounds__(BLOCK, queue_min_blocks<ALGO, BLOCK>())
    bin_kernel(const FoldParams p) {
    if constexpr (PERSIST) {
        for_each_queued_item<BLOCK * ROUNDS>(p, [&](const WorkItem& w, uint32_t k) {
            bin_item<ALGO, CNT16, BLOCK, REF_STATS, ROUNDS>(p, w, k);
        });
    } else {
        bin_item<ALGO, CNT16, BLOCK, REF_STATS, ROUNDS>(
            p, queue_item<BLOCK * ROUNDS>(p, blockIdx.x), blockIdx.x);
    }
}

// CE per-point bin data for bin_kernel: {counter word of the magnitude
// column within a phase row, increment}.  The kernel turns the word into a
// byte offset for its CTA shape when it stages the tile, so the data serves
// every block size the autotuner tries.
__global__ void ce_binaux_kernel(const float* __restrict__ m, uint2* __restrict__ aux,
                                 const CurveDesc* __restrict__ curves, uint32_t n_curves,
                                 uint32_t n_mag, float mag_bin_size, int cnt16) {
    const uint32_t c = blockIdx.x;
    if (c >= n_curves) return;
    const CurveDesc cd = curves[c];
    const uint32_t n4 = (cd.n + 3u) & ~3u;
    for (uint32_t i = threadIdx.x; i < n4; i += blockDim.x) {
        uint2 v = make_uint2(0u, 0u);
        if (i < cd.n) {
            const float mag_val = m[cd.off + i];
            // MagBin (periodfind/cuda/ce.cu:70-72; rust/src/ce.rs:79).
            const unsigned long long mb64 =
                static_cast<unsigned long long>(mag_val / mag_bin_size);
            const uint32_t mb = (uint32_t)(mb64 % n_mag);
            if (cnt16) {
                v.x = mb >> 1;
                v.y = (mb & 1u) ? 0x10000u : 1u;
            } else {
                v.x = mb;
                v.y = 1u;
            }
        }
        aux[cd.off + i] = v;
    }
}

}  // namespace PF_KNS
}  // namespace pfk
