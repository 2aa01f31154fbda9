// pf_types.h -- device data layout shared by the host driver and the kernels.
#pragma once
#include <stddef.h>
#include <stdint.h>

namespace pfk {

enum : int { ALGO_CE = 0, ALGO_AOV = 1, ALGO_LS = 2 };

// Fold variants.  REF: the reference expression with an FP64 divide per
// (point, period) (periodfind/cuda/ce.cu:141-143).  EXACT: the same
// correctly-rounded quotient from a per-period double-double reciprocal
// (bit-identical results, no divide).  DF: split-precision FP32 phase
// frac(t * f) (LS only).  F32: the whole fold in FP32 (precision study).
enum : int { FOLD_REF = 0, FOLD_EXACT = 1, FOLD_DF = 2, FOLD_F32 = 3 };

// AOV accumulation.  F32: per-bin (count, sum, sum of squares) with f32
// adds in point order, as the reference.  FIX: one 64-bit integer per bin
// holding (count << 44) + sum of fixed-point magnitudes; exact and order
// independent; statistic finished in FP64.
enum : int { AOVACC_F32 = 0, AOVACC_FIX = 1 };

constexpr int kFixCountShift = 44;

constexpr uint32_t kTile = 1024;     // points staged per tile (multiple of 4)
constexpr uint32_t kBinTile = 256;   // points per tile in the chosen bin kernel

// One light curve in the packed arrays.  Curves start on 16-byte
// boundaries (offsets are multiples of 4 points).
struct CurveDesc {
    int64_t off;     // first point in the packed arrays
    uint32_t n;      // number of points
    float avg;       // AOV: f32 sequential mean of the magnitudes
    double fix_mn;   // AOV FIX: magnitude offset (curve minimum)
    double fix_scale;  // AOV FIX: fixed-point units per magnitude unit
    double fix_sumx;   // AOV FIX: sum of fixed-point magnitudes
    double fix_sumx2;  // AOV FIX: sum of squared fixed-point magnitudes
};

// One CTA's share of the work: `np` consecutive trial periods starting at
// `p0`, one period derivative `pdt`, one curve.  A CTA never mixes period
// derivatives, so the derivative branch is uniform.
struct WorkItem {
    uint32_t curve;
    uint32_t pdt;
    uint32_t p0;
    uint32_t np;
};

// Device work queue of the persistent (chosen-form) kernels.  Item k of a
// launch is curve order[k / (n_pdt * tiles)], then period derivative and
// tile of BLOCK consecutive periods from the remainder (tiles =
// ceil(n_per / BLOCK)); CTAs take items from *next, which is zeroed before
// the launch.  `order` lists the curves longest first, so the long items
// start first and the short ones fill the tail.
struct WorkQueue {
    const uint32_t* order;
    uint32_t n_work;
    unsigned* next;
};

struct FoldParams {
    const float* t;          // packed times
    const float* m;          // packed magnitudes (AOV F32, LS)
    const uint32_t* aux32;   // CE: packed magnitude bin per point
    const uint64_t* aux64;   // AOV FIX: packed (1 << 44) + fixed-point mag
    const CurveDesc* curves;
    const WorkItem* work;
    const float* periods;
    const float* pdts;
    float* out;              // [curve][n_per][n_pdt]
    uint32_t n_per, n_pdt;
    uint32_t n_phase, n_mag, p_overlap, m_overlap;
    float phase_bin_size, mag_bin_size;
    const unsigned* tmax_bits;  // float bits of max |t| over the batch
    uint32_t edge_d;            // bin-edge guard (units of 2^-20 of a bin)
    unsigned long long* stamps; // optional: [work item][start, end] globaltimer ns
    WorkQueue q;                // persistent kernels (instead of `work`)
    // Optional (occupancy tests): raw bin counts per cell, [curve][n_per]
    // [n_pdt][bins] with bins = n_phase * n_mag (CE) or n_phase (AOV).
    // Written by the plain kernels and the chosen reference-statistic form.
    uint32_t* bins;
    // LS on a uniform frequency grid (fgrid != 0): trial frequency k is
    // f0 + k * df exactly (FP64), in place of 1 / periods[k]; one period
    // derivative, 0.
    int fgrid;
    double f0, df;
};

// Shared-memory bytes of the chosen bin kernel (pf_bin.cuh).
inline size_t bin_smem_bytes(int algo, bool cnt16, int block, uint32_t n_phase,
                             uint32_t n_mag) {
    size_t bytes = (size_t)kBinTile * 16;  // {double t; u32 a, b} per point
    if (algo == ALGO_CE) {
        const size_t w = cnt16 ? (n_mag + 1) / 2 : n_mag;
        bytes += (size_t)n_phase * w * block * 4;
    } else {
        bytes += (size_t)2 * n_phase * block * 4;
    }
    return bytes;
}

// Shared-memory bytes for one CTA (host and device agree through this).
inline size_t fold_smem_bytes(int algo, int fold, int acc, int block,
                                                  bool ovl, uint32_t n_phase,
                                                  uint32_t n_mag) {
    size_t tt = (fold == FOLD_EXACT) ? 8 : 4;
    size_t ta = (algo == ALGO_AOV && acc == AOVACC_FIX) ? 8 : 4;
    size_t bytes = kTile * (tt + ta);
    if (algo == ALGO_CE) {
        size_t slots = (size_t)(ovl ? n_phase : n_phase + 1) * n_mag;
        bytes += slots * block * 4;
    } else if (algo == ALGO_AOV) {
        if (acc == AOVACC_FIX) {
            bytes += (size_t)(ovl ? n_phase : n_phase + 1) * block * 8;
        } else {
            bytes += (size_t)n_phase * block * 12;
        }
    }
    return bytes;
}

}  // namespace pfk
