// pf_fpw.cuh -- FPW (fast phase-folding weighted) and BLS periodograms, included by
// each arithmetic unit after pf_fold.cuh and pf_bin.cuh.
//
// Statistic (rust/src/fpw.rs:12-66; periodfind/cuda/fpw.cu:45-224): each
// point carries an inverse variance w = 1 / err^2 and w * m; the fold puts
// it in one of n_bins phase bins; per bin V = sum w, Y = sum w * m; the
// value is sum over bins with V > 0 of Y^2 / (2 V).  Maximum is best.
//
// Decomposition: a CTA per (curve, period derivative, tile of BLOCK trial
// periods); thread j owns one period for the whole curve and keeps its own
// V and Y in shared memory ([bin][thread], so a warp's updates touch
// consecutive words: the chosen form as (V, Y) float2 pairs, one 8-byte
// access per update; the plain form as V rows then Y rows), adding the
// points in curve order -- the Rust path's order, so the sums round as it
// does.  The curve streams through shared memory in 16-byte point records,
// 256 points per tile.
//
// The bin is the reference's for the unit's semantics:
//   CUDA build: (size_t)(folded / bin_size), clamped to n_bins - 1
//               (fpw.cu:28-30, 115-117);
//   Rust path:  (folded * n_bins) as usize, clamped (fpw.rs:44);
// with folded = (float)|q - floor(q)| for the correctly rounded quotient q.
//
// Plain form: that sequence for every point (FP64 divide).  Chosen form: the
// bin from q' = t * RN(1/P) with a round-down floor and one round-down FMA
// that yields floor(q' n_bins) and 20 fraction bits (the chosen CE / AOV bin
// kernel's construction); a point whose fraction lies within the proven
// guard of a bin edge takes the reference sequence instead (divide-free, the
// same quotient).  Unlike the integer CE / AOV counters, float sums cannot
// take a point back, so each point is tested before it is added.
#pragma once

#ifndef PF_KNS
#error "include after defining PF_KNS"
#endif

namespace pfk {
namespace PF_KNS {

constexpr uint32_t kFpwTile = 256;

// The reference's bin of a folded phase, with this unit's arithmetic.
__device__ __forceinline__ uint32_t fpw_ref_bin(float folded, const FpwParams& p) {
#if PF_SEM_CPU_TU
    const uint32_t b = trunc_u(folded * (float)p.n_bins);
#else
    const uint32_t b = trunc_u(folded / p.bin_size);
#endif
    return min(b, p.n_bins - 1u);
}

// BLS (Box Least Squares, rust/src/bls.rs:19-134; periodfind/cuda/bls.cu:
// 56-308) shares the binning: the second sum is w * (m - weighted mean), the
// bins sit one row down so that row 0 holds the zero of the prefix sums, and
// the value is the best s^2 / (r (W - r)) over the windows of nb_min ..
// nb_max consecutive bins (wrapping) whose weight fraction r / W lies in
// (0, 1); 0 when W <= 0.
template <int BLOCK, bool CHOSEN, bool BLS, int GROUP>
__global__ void __launch_bounds__(BLOCK)
    fpw_kernel(const FpwParams p, uint32_t tiles_per_row) {
    using TT = typename std::conditional<CHOSEN, double, float>::type;
    // One 16-byte record per staged point: a single 128-bit shared load.
    struct alignas(16) Point {
        TT t;
        float iv, ivy;
    };
    constexpr uint32_t kRow0 = BLS ? 1u : 0u;  // rows before bin 0
    extern __shared__ __align__(16) unsigned char fsm[];
    Point* st = reinterpret_cast<Point*>(fsm);
    // Per-thread bins, row k (bin k - kRow0) of thread tid: the chosen form
    // keeps (V, Y) pairs, [row][BLOCK] float2, so a bin update is one 8-byte
    // load and store; the plain form keeps V rows then Y rows.
    float* bins = reinterpret_cast<float*>(st + kFpwTile);
    const uint32_t rows = p.n_bins + kRow0;
    auto ld = [&](uint32_t k) -> float2 {
        if constexpr (CHOSEN)
            return reinterpret_cast<const float2*>(bins)[k * BLOCK + threadIdx.x];
        else
            return make_float2(bins[k * BLOCK + threadIdx.x], bins[(rows + k) * BLOCK + threadIdx.x]);
    };
    auto put = [&](uint32_t k, float2 x) {
        if constexpr (CHOSEN) {
            reinterpret_cast<float2*>(bins)[k * BLOCK + threadIdx.x] = x;
        } else {
            bins[k * BLOCK + threadIdx.x] = x.x;
            bins[(rows + k) * BLOCK + threadIdx.x] = x.y;
        }
    };
    __shared__ double warp_min[BLOCK / 32];

    const uint64_t cta = blockIdx.x;
    const uint32_t tile = (uint32_t)(cta % tiles_per_row);
    const uint64_t row = cta / tiles_per_row;     // curve * n_pdt + pdt
    const uint64_t c = row / p.n_pdt;
    const uint32_t d = (uint32_t)(row % p.n_pdt);
    const int tid = threadIdx.x;
    const uint64_t pi = (uint64_t)tile * BLOCK + tid;
    const bool active = pi < p.n_per;

    const int64_t off = p.off[c];
    const uint32_t n = p.len[c];
    const uint32_t nb = p.n_bins;
    for (uint32_t k = 0; k < rows; k++) put(k, make_float2(0.0f, 0.0f));
    const float period = p.periods[active ? pi : (uint64_t)tile * BLOCK];
    const float period_dt = p.pdts[d];
    Cell s;
    cell_setup<CHOSEN ? FOLD_EXACT : FOLD_REF>(s, period, period_dt);
    const bool has_pdt = period_dt != 0.0f;

    // Chosen form: the fast bin is exact away from bin edges while
    // |q| * n_bins < 2^30 (the same bound as the chosen CE / AOV kernels),
    // checked for the CTA from max|t| and its smallest |P|.
    bool fast = false, fast32 = false;
    if constexpr (CHOSEN) {
        double mn = fabs((double)period);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        if ((tid & 31) == 0) warp_min[tid >> 5] = mn;
        __syncthreads();
        double pmin = warp_min[0];
#pragma unroll
        for (int k = 1; k < BLOCK / 32; k++) pmin = fmin(pmin, warp_min[k]);
        const double qb = p.tmax / pmin + fabs((double)period_dt) * p.tmax * p.tmax /
                                              (2.0 * pmin * pmin);
        fast = qb * (double)nb < 1073741824.0;  // 2^30
        // |q| < 2^19 as well: the one-FMA bin below.
        fast32 = fast && qb < 524288.0;
    }
    const double nd20 = (double)nb * 1048576.0;
    const uint32_t n_neg = 0u - nb;
    const uint32_t edge_add = p.edge_d << 12;
    const uint32_t edge_lim = (2u * p.edge_d) << 12;
    // The guard in units of 2^-32 of a bin, widened by n_bins + 2 units for
    // the truncation of the phase to 32 bits.
    const uint32_t edge32_add = edge_add + nb + 2u;
    const uint32_t edge32_lim = 2u * edge32_add;
    const double y32 = s.yhi * 4294967296.0;  // RN(1/P) * 2^32, exact

    // The reference's bin of point time t (the fast bin when the CTA's
    // bound allows, the reference sequence near an edge or otherwise).
    auto bin_of = [&](TT t) -> uint32_t {
        if constexpr (CHOSEN) {
            const double td = t;
            if (fast32) {
                // One FMA on the exact product t * (RN(1/P) * 2^32) leaves
                // floor(frac(q') * 2^32) in the low word f; the 64-bit
                // product f * n_bins holds the bin (high word) and the
                // position within it (low word, for the edge test).
                const double a = has_pdt ? td - s.c * td * td : td;
                const double y = __fma_rd(a, y32, kMagic15);
                const uint32_t f = (uint32_t)__double2loint(y);
                const unsigned long long fn = (unsigned long long)f * nb;
                if ((uint32_t)fn + edge32_add >= edge32_lim) return (uint32_t)(fn >> 32);
            } else if (fast) {
                const double a = has_pdt ? td - s.c * td * td : td;
                const double qh = __dmul_rn(a, s.yhi);
                const double r = __dadd_rd(qh, kMagic15);
                const double y = __fma_rd(qh, nd20, kMagic15);
                const uint32_t ylo = (uint32_t)__double2loint(y);
                const uint32_t yhi = (uint32_t)__double2hiint(y);
                // floor(q' n_bins) - n_bins floor(q'), biased by 2^31 by the
                // magic constant's top mantissa bit.
                const uint32_t b = __funnelshift_r(ylo, yhi, 20) +
                                   (uint32_t)__double2loint(r) * n_neg - 0x80000000u;
                if (ylo * 4096u + edge_add >= edge_lim) return b;
            }
            return fpw_ref_bin(has_pdt ? fold_exact<true>(td, s) : fold_exact<false>(td, s), p);
        } else {
            return fpw_ref_bin(fold_ref(t, s), p);
        }
    };

    for (uint32_t base = 0; base < n; base += kFpwTile) {
        const uint32_t cnt = min(kFpwTile, n - base);
        __syncthreads();
        for (uint32_t i = tid; i < cnt; i += BLOCK)
            st[i] = Point{(TT)p.t[off + base + i], p.iv[off + base + i], p.ivy[off + base + i]};
        __syncthreads();
        if (!active) continue;
        uint32_t i = 0;
        if constexpr (GROUP > 1) {
            // GROUP points are read and binned before the first of their
            // read-modify-writes: the staged tile and the bins share one
            // shared-memory array, so a point read cannot move above an
            // earlier bin store, and one point at a time would chain the
            // point read, the bin arithmetic and the bin update per point.
            // The updates stay in point order (same bin, same rounding).
            for (; i + GROUP <= cnt; i += GROUP) {
                Point q[GROUP];
                uint32_t b[GROUP];
#pragma unroll
                for (int k = 0; k < GROUP; k++) q[k] = st[i + k];
#pragma unroll
                for (int k = 0; k < GROUP; k++) b[k] = bin_of(q[k].t);
#pragma unroll
                for (int k = 0; k < GROUP; k++) {
                    float2 x = ld(b[k] + kRow0);
                    x.x += q[k].iv;
                    x.y += q[k].ivy;
                    put(b[k] + kRow0, x);
                }
            }
        }
#pragma unroll 4
        for (; i < cnt; i++) {
            const Point pt = st[i];
            const uint32_t bin = bin_of(pt.t);
            float2 x = ld(bin + kRow0);
            x.x += pt.iv;
            x.y += pt.ivy;
            put(bin + kRow0, x);
        }
    }
    if (!active) return;
    float acc = 0.0f;
    if constexpr (BLS) {
        // Prefix sums in place, in the reference's order (bls.rs:83-89):
        // row k + 1 becomes row k + row k + 1.
        float2 prev = ld(0);
        for (uint32_t k = 0; k < nb; k++) {
            float2 x = ld(k + 1);
            x.x = prev.x + x.x;
            x.y = prev.y + x.y;
            put(k + 1, x);
            prev = x;
        }
        const float w_total = prev.x, y_total = prev.y;
        if (w_total > 0.0f) {
            // Every (phase, width) window, phase-major: the window's start
            // row is read once per phase.  The sums are the reference's:
            // end <= nb gives row[end] - row[phi] (x - y is x + (-y)
            // exactly), a wrapping window (total - row[phi]) + row[end - nb];
            // the maximum does not depend on the order of the windows.
            for (uint32_t phi = 0; phi < nb; phi++) {
                const float2 a = ld(phi);
                const float w_rest = w_total - a.x, y_rest = y_total - a.y;
                for (uint32_t nbw = p.nb_min; nbw <= p.nb_max; nbw++) {
                    const uint32_t end = phi + nbw;
                    const bool wrap = end > nb;
                    const float2 e = ld(wrap ? end - nb : end);
                    const float r = e.x + (wrap ? w_rest : -a.x);
                    const float sy = e.y + (wrap ? y_rest : -a.y);
                    const float r_frac = r / w_total;
                    if (r_frac > 0.0f && r_frac < 1.0f) {
                        const float bls = (sy * sy) / (r * (w_total - r));
                        if (bls > acc) acc = bls;
                    }
                }
            }
        }
    } else {
        for (uint32_t k = 0; k < nb; k++) {
            const float2 x = ld(k);
            if (x.x > 0.0f) acc += x.y * x.y / (2.0f * x.x);
        }
    }
    p.out[(uint64_t)c * (p.n_per * p.n_pdt) + pi * p.n_pdt + d] = acc;
}

}  // namespace PF_KNS
}  // namespace pfk
