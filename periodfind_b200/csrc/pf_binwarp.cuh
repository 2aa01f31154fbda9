// pf_binwarp.cuh -- the chosen CE / AOV binning with shared histograms and
// shared-memory atomics: the other strategy the autotuner weighs against
// per-thread privatised histograms (pf_bin.cuh).
//
// Included by the two semantics units after pf_bin.cuh (same namespace).
//
// The reference switches strategy on curve length (periodfind/cuda/aov.cu:
// 73-132 atomic shared bins, :133-211 per-thread private arrays).  Here the
// privatised form gives every thread its own trial period and its own
// histogram; this form gives a warp one histogram per trial period: the 32
// lanes take different points of the curve and add them into the warp's
// histogram with shared atomics (red.shared, colliding lanes serialised by
// the hardware), then the warp finishes the statistic together, one phase
// row (CE) or bin (AOV) per lane.  A warp works through 32 periods of its
// item one after the other; the whole curve is staged in shared memory once
// per item, so the form serves curves of up to kWarpMaxPoints points.
//
// Bins come from the same fast FP64 / integer arithmetic with the reference
// sequence near bin edges as the privatised form, so the occupancies are
// identical; the statistic adds the same terms in the same order (the row or
// bin terms in parallel, their running sum by lane 0 in row order), so the
// values are bit-identical to the privatised form's.
#pragma once

namespace pfk {
namespace PF_KNS {

// Shared memory of one CTA: the staged curve, then one histogram per warp
// (CE n_phase x n_mag u32 counts; AOV n_phase counts and n_phase
// fixed-point sums).
__host__ __device__ constexpr size_t binwarp_smem_bytes(int algo, int block, uint32_t n_phase,
                                                        uint32_t n_mag) {
    return (size_t)kWarpMaxPoints * 16 +
           (size_t)(block / 32) * (algo == ALGO_CE ? n_phase * n_mag : 2 * n_phase) * 4;
}

template <int ALGO, int BLOCK>
__device__ __forceinline__ void binwarp_item(const FoldParams& p, const WorkItem w,
                                             uint32_t item) {
    extern __shared__ __align__(16) unsigned char smem[];
    BinPoint* tile = reinterpret_cast<BinPoint*>(smem);
    stamp_start(p, item);
    const CurveDesc cd = p.curves[w.curve];
    const uint32_t n = cd.n;  // <= kWarpMaxPoints (the host offers the form only then)
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const float period_dt = p.pdts[w.pdt];
    const uint32_t nP = p.n_phase, nM = p.n_mag;
    const uint32_t hist_words = (ALGO == ALGO_CE) ? nP * nM : 2 * nP;
    uint32_t* hist =
        reinterpret_cast<uint32_t*>(smem + (size_t)kWarpMaxPoints * 16) + warp * hist_words;
    const uint32_t hist_base = (uint32_t)__cvta_generic_to_shared(hist);

    // Range guard over every period of the item, as the privatised form.
    const uint32_t jt = (uint32_t)tid;
    const float per_t = p.periods[w.p0 + (jt < w.np ? jt : 0u)];
    const bool fin = isfinite(period_dt) && isfinite(per_t) && per_t != 0.0f;
    const double qb = cta_qbound_of<BLOCK>(p, fabs((double)per_t), period_dt);
    const bool fast = __syncthreads_and(fin ? 1 : 0) && qb * (double)nP < 1073741824.0;

    // Stage the curve: t as a double; CE: the magnitude bin; AOV: the
    // fixed-point magnitude.
    for (uint32_t i4 = tid; i4 < (n + 3) / 4; i4 += BLOCK) {
        const float4 q = reinterpret_cast<const float4*>(p.t + cd.off)[i4];
        const float tq[4] = {q.x, q.y, q.z, q.w};
        if constexpr (ALGO == ALGO_CE) {
            // The prepared CE data is (16-bit counter word, increment):
            // magnitude bin = 2 * word + (increment == 1 << 16).
            const uint4 a01 = reinterpret_cast<const uint4*>(p.aux64 + cd.off)[2 * i4];
            const uint4 a23 = reinterpret_cast<const uint4*>(p.aux64 + cd.off)[2 * i4 + 1];
            const uint32_t mb[4] = {2 * a01.x + (a01.y >> 16), 2 * a01.z + (a01.w >> 16),
                                    2 * a23.x + (a23.y >> 16), 2 * a23.z + (a23.w >> 16)};
#pragma unroll
            for (int k = 0; k < 4; k++) tile[4 * i4 + k] = BinPoint{(double)tq[k], mb[k], 0u};
        } else {
            const uint4 a = reinterpret_cast<const uint4*>(p.aux32 + cd.off)[i4];
            const uint32_t fx[4] = {a.x, a.y, a.z, a.w};
#pragma unroll
            for (int k = 0; k < 4; k++) tile[4 * i4 + k] = BinPoint{(double)tq[k], fx[k], 0u};
        }
    }
    __syncthreads();

    const double nd20 = (double)nP * 1048576.0;
    const uint32_t n_neg = 0u - nP;
    const uint32_t edge_add = p.edge_d << 12;
    const uint32_t edge_lim = (2u * p.edge_d) << 12;

    for (uint32_t q = 0; q < 32u; q++) {
        const uint32_t j = (uint32_t)warp * 32u + q;
        if (j >= w.np) break;  // uniform over the warp
        const uint32_t pi = w.p0 + j;
        Cell s;
        cell_setup<FOLD_EXACT>(s, p.periods[pi], period_dt);
        for (uint32_t k = lane; k < hist_words; k += 32) hist[k] = 0u;
        __syncwarp();
        // The bin of one point: the fast form, or the reference sequence
        // within the edge guard (as pf_bin.cuh's fast_bin / exact_bin).
        auto bin_of = [&](double td, auto has_pdt_tag) -> uint32_t {
            constexpr bool HAS_PDT = decltype(has_pdt_tag)::value;
            if (fast) {
                const double a = HAS_PDT ? td - s.c * td * td : td;
                const double qh = __dmul_rn(a, s.yhi);
                const double r = __dadd_rd(qh, kMagic15);
                const double y = __fma_rd(qh, nd20, kMagic15);
                const uint32_t ylo = (uint32_t)__double2loint(y);
                const uint32_t yhi = (uint32_t)__double2hiint(y);
                const uint32_t ev = ylo * 4096u + edge_add;
                if (ev >= edge_lim)
                    return (__funnelshift_r(ylo, yhi, 20) + (uint32_t)__double2loint(r) * n_neg) -
                           0x80000000u;
            }
            const float folded = fold_exact<HAS_PDT>(td, s);
            const uint32_t pb = min(trunc_u(folded / p.phase_bin_size), nP);
            return pb == nP ? 0u : pb;
        };
        auto run = [&](auto has_pdt_tag) {
            for (uint32_t i = lane; i < n; i += 32) {
                const uint4 raw = reinterpret_cast<const uint4*>(tile)[i];
                const double td = __hiloint2double((int)raw.y, (int)raw.x);
                const uint32_t row = bin_of(td, has_pdt_tag);
                if constexpr (ALGO == ALGO_CE) {
                    red_shared_u32(hist_base + (row * nM + raw.z) * 4u, 1u);
                } else {
                    red_shared_u32(hist_base + row * 4u, 1u);
                    red_shared_u32(hist_base + (nP + row) * 4u, raw.z);
                }
            }
        };
        if (period_dt != 0.0f) run(std::true_type{});
        else run(std::false_type{});
        compiler_fence();
        __syncwarp();

        // The statistic: each lane one phase row (CE) or bin (AOV) term, in
        // the privatised form's operation order; lane 0 adds them in order.
        const size_t out_idx =
            (size_t)w.curve * ((size_t)p.n_per * p.n_pdt) + (size_t)pi * p.n_pdt + w.pdt;
        if constexpr (ALGO == ALGO_CE) {
            float acc = 0.0f;
            for (uint32_t j0 = 0; j0 < nP; j0 += 32) {
                const uint32_t jr = j0 + (uint32_t)lane;
                float term = 0.0f;
                if (jr < nP) {
                    uint32_t col = 0;
                    float row = 0.0f;
                    // Pairs of magnitude bins, as the privatised form's
                    // 16-bit packed words.
                    for (uint32_t i = 0; i < nM; i += 2) {
                        const uint32_t c0 = hist[jr * nM + i];
                        const uint32_t c1 = (i + 1 < nM) ? hist[jr * nM + i + 1] : 0u;
                        col += c0 + c1;
                        row = __fadd_rn(row, __fadd_rn(ce_xlx(c0), ce_xlx(c1)));
                    }
                    term = __fsub_rn(ce_xlx(col), row);
                }
                const uint32_t cnt = min(32u, nP - j0);
                for (uint32_t l = 0; l < cnt; l++)
                    acc = __fadd_rn(acc, __shfl_sync(0xffffffffu, term, (int)l));
            }
            if (lane == 0) p.out[out_idx] = ce_finish(acc, n);
        } else {
            double sbx = 0.0;
            for (uint32_t b0 = 0; b0 < nP; b0 += 32) {
                const uint32_t b = b0 + (uint32_t)lane;
                double x2 = 0.0, rc = 0.0;
                if (b < nP) {
                    const uint32_t c = hist[b];
                    const double Xd = (double)hist[nP + b];
                    x2 = __dmul_rn(Xd, Xd);
                    rc = __drcp_rn((double)max(c, 1u));
                }
                const uint32_t cnt = min(32u, nP - b0);
                for (uint32_t l = 0; l < cnt; l++)
                    sbx = __fma_rn(__shfl_sync(0xffffffffu, x2, (int)l),
                                   __shfl_sync(0xffffffffu, rc, (int)l), sbx);
            }
            if (lane == 0) p.out[out_idx] = aov_finish(sbx, cd, n, nP);
        }
        __syncwarp();
    }
    stamp_end(p, item);
}

// Items from the device work queue (BLOCK periods each; a warp takes 32 of
// them), persistently or one CTA per item.
template <int ALGO, int BLOCK, bool PERSIST>
__global__ void __launch_bounds__(BLOCK) binwarp_kernel(const FoldParams p) {
    if constexpr (PERSIST) {
        for_each_queued_item<BLOCK>(p, [&](const WorkItem& w, uint32_t k) {
            binwarp_item<ALGO, BLOCK>(p, w, k);
        });
    } else {
        binwarp_item<ALGO, BLOCK>(p, queue_item<BLOCK>(p, blockIdx.x), blockIdx.x);
    }
}

}  // namespace PF_KNS
}  // namespace pfk
