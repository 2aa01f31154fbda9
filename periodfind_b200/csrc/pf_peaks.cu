// pf_peaks.cu -- top-N peak search over periodograms on the device.
//
// Semantics of rust/src/peaks.rs:18-238 (find_top_peaks on one chunk): the
// interior samples 1 .. n-2 of the flattened [period][pdt] grid are fed in
// order; a strict local extremum that beats the current threshold (the
// worst of the top-N once it is full) becomes the candidate unless a better
// candidate is pending; the candidate is promoted into the best-first list
// once min_distance samples have been fed since it was set, and at the end.
//
// Only extrema change the state; every other sample just advances the
// distance counter.  A CTA per curve therefore (1) flags extrema in chunks,
// (2) compacts them in index order with a block scan, and (3) one thread
// replays the state machine over the compacted extrema, reconstructing the
// distance counter from index gaps:
//   - a candidate set at index c is promoted while feeding index
//     c + min_distance - 1 (after that index's own peak test), or at the
//     end if no such index is fed;
//   - a better extremum fed before that replaces it.
// The sorted top-N list lives in shared memory (threshold in a register)
// and is written to the caller's rows at the end.  Lists of at most 32
// peaks take peaks_warp_kernel instead: a warp per curve holds the list
// across its lanes and does the flagging, compaction and replay itself.
// (Both kernels give the same results: the state machine is the same and
// only the chunking of the extrema differs.)
//
// Extrema that cannot pass the peak test are dropped before the replay.
// The threshold only ever gets stricter (a full list only takes a better
// value in place of its worst), so an extremum that is not better than the
// threshold at the start of its chunk fails the peak test at its own turn
// too.  Such an extremum changes no state: a promotion that falls due while
// it would be fed depends only on the candidate and the threshold, so it
// gives the same list when done at the next extremum that is fed instead.
// On noisy rows this leaves a few hundred of the ~n/3 extrema to replay.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "pf_launch.h"

namespace pfk {

namespace {

constexpr int kPeakThreads = 256;
constexpr int kPerThread = 8;
constexpr uint32_t kChunk = kPeakThreads * kPerThread;

struct PeakState {
    int64_t* idx;   // shared memory, n_peaks entries
    float* val;
    uint32_t count, n_peaks;
    bool use_max;
    bool has_cand;
    int64_t cand_idx;
    float cand_val;
    float thr;      // threshold(): the worst kept value once the list is full
};

__device__ __forceinline__ bool better(bool use_max, float a, float b) {
    return use_max ? (a > b) : (a < b);
}

// peaks.rs:104-130: append (or replace the worst) and bubble toward the front.
__device__ void insert(PeakState& s, int64_t idx, float v) {
    uint32_t i;
    if (s.count < s.n_peaks) {
        i = s.count++;
    } else if (better(s.use_max, v, s.val[s.count - 1])) {
        i = s.count - 1;
    } else {
        return;
    }
    s.idx[i] = idx;
    s.val[i] = v;
    while (i > 0 && better(s.use_max, s.val[i], s.val[i - 1])) {
        const float tv = s.val[i];
        s.val[i] = s.val[i - 1];
        s.val[i - 1] = tv;
        const int64_t ti = s.idx[i];
        s.idx[i] = s.idx[i - 1];
        s.idx[i - 1] = ti;
        i--;
    }
    if (s.count == s.n_peaks) s.thr = s.val[s.count - 1];
}

// peaks.rs:134-140.
__device__ __forceinline__ void promote(PeakState& s) {
    if (s.has_cand && better(s.use_max, s.cand_val, s.thr)) insert(s, s.cand_idx, s.cand_val);
    s.has_cand = false;
}

// The same list and candidate for n_peaks <= 32, held across one warp: lane
// k keeps entry k, and every lane keeps the same copy of the rest of the
// state.  An insertion takes the new entry's place from one ballot (the
// entries not strictly worse stay ahead, which is where peaks.rs's bubble
// stops) and shifts the entries behind it down one lane.
struct WarpTop {
    int64_t idx;  // this lane's entry
    float val;
    uint32_t count, n_peaks;
    bool use_max;
    bool has_cand;
    int64_t cand_idx;
    float cand_val;
    float thr;
};

__device__ __forceinline__ void warp_insert(WarpTop& w, int lane, int64_t idx, float v) {
    constexpr unsigned kAll = 0xffffffffu;
    if (w.count == w.n_peaks &&
        !better(w.use_max, v, __shfl_sync(kAll, w.val, (int)w.count - 1)))
        return;
    const bool ahead = lane < (int)w.count && !better(w.use_max, v, w.val);
    const int pos = __popc(__ballot_sync(kAll, ahead));
    const int64_t up_idx = __shfl_up_sync(kAll, w.idx, 1);
    const float up_val = __shfl_up_sync(kAll, w.val, 1);
    if (lane == pos) {
        w.idx = idx;
        w.val = v;
    } else if (lane > pos) {
        w.idx = up_idx;
        w.val = up_val;
    }
    if (w.count < w.n_peaks) w.count++;
    if (w.count == w.n_peaks) w.thr = __shfl_sync(kAll, w.val, (int)w.n_peaks - 1);
}

__device__ __forceinline__ void warp_promote(WarpTop& w, int lane) {
    if (w.has_cand && better(w.use_max, w.cand_val, w.thr))
        warp_insert(w, lane, w.cand_idx, w.cand_val);
    w.has_cand = false;
}

// Dynamic shared memory: [kChunk int64 extrema indices][kChunk f32 values]
// [n_peaks int64][n_peaks f32] (the best-first list).
// The streaming state machine over one chunk's compacted extrema (index
// order), by one warp holding the top list across its lanes: extrema that
// do not beat the threshold are skipped by ballot, the others fed in turn
// (peaks.rs:18-238: promotion of a due candidate, candidate replacement,
// promotion once min_distance samples have been fed).
__device__ __forceinline__ void warp_replay(WarpTop& w, int lane, const int64_t* ext_idx,
                                            const float* ext_val, uint32_t ne, uint64_t md,
                                            bool use_max) {
    for (uint32_t b0 = 0; b0 < ne; b0 += 32) {
        const uint32_t e = b0 + lane;
        const bool in = e < ne;
        const int64_t my_i = in ? ext_idx[e] : 0;
        const float my_v = in ? ext_val[e] : 0.0f;
        uint32_t pending =
            __ballot_sync(0xffffffffu, in && better(use_max, my_v, w.thr));
        while (pending) {
            const int k = __ffs(pending) - 1;
            const int64_t i = __shfl_sync(0xffffffffu, my_i, k);
            const float v = __shfl_sync(0xffffffffu, my_v, k);
            if (w.has_cand && (uint64_t)w.cand_idx + (md > 0 ? md - 1 : 0) <
                                  (uint64_t)i)
                warp_promote(w, lane);
            if (better(use_max, v, w.thr) &&
                (!w.has_cand || better(use_max, v, w.cand_val))) {
                w.cand_idx = i;
                w.cand_val = v;
                w.has_cand = true;
            }
            if (w.has_cand && (uint64_t)(i - w.cand_idx) + 1 >= md)
                warp_promote(w, lane);
            pending &= ~(1u << k);
            pending &= __ballot_sync(0xffffffffu, better(use_max, my_v, w.thr));
        }
    }
}

__global__ void __launch_bounds__(kPeakThreads)
    peaks_kernel(const float* __restrict__ pg, uint64_t flat_len, uint32_t n_peaks,
                 uint32_t min_distance, int use_max_i, int64_t* __restrict__ out_idx,
                 float* __restrict__ out_val) {
    extern __shared__ __align__(16) unsigned char psmem[];
    int64_t* ext_idx = reinterpret_cast<int64_t*>(psmem);
    float* ext_val = reinterpret_cast<float*>(psmem + kChunk * 8);
    int64_t* top_idx = reinterpret_cast<int64_t*>(psmem + kChunk * 12);
    float* top_val = reinterpret_cast<float*>(psmem + kChunk * 12 + (size_t)n_peaks * 8);
    __shared__ uint32_t warp_tot[kPeakThreads / 32];
    __shared__ uint32_t chunk_count;
    __shared__ float thr_sh;  // the replay's threshold after the last chunk

    const uint64_t c = blockIdx.x;
    const float* d = pg + c * flat_len;
    const bool use_max = use_max_i != 0;

    const bool warp_list = n_peaks <= 32;
    WarpTop w;
    w.idx = -1;
    w.val = 0.0f;
    w.count = 0;
    w.n_peaks = n_peaks;
    w.use_max = use_max;
    w.has_cand = false;
    w.cand_idx = -1;
    w.cand_val = use_max ? -INFINITY : INFINITY;
    w.thr = use_max ? -INFINITY : INFINITY;

    PeakState s;
    s.idx = top_idx;
    s.val = top_val;
    s.count = 0;
    s.n_peaks = n_peaks;
    s.use_max = use_max;
    s.has_cand = false;
    s.cand_idx = -1;
    s.cand_val = use_max ? -INFINITY : INFINITY;
    s.thr = use_max ? -INFINITY : INFINITY;
    const uint64_t md = min_distance;

    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) thr_sh = s.thr;
    __syncthreads();
    // Interior samples 1 .. flat_len-2.
    const uint64_t first = 1, last = (flat_len >= 2) ? flat_len - 2 : 0;
    for (uint64_t base = first; flat_len >= 3 && base <= last; base += kChunk) {
        // (1) flag this thread's kPerThread consecutive samples: strict
        // extrema better than the threshold at the start of the chunk.
        uint32_t flags = 0;
        const uint64_t i0 = base + (uint64_t)tid * kPerThread;
        const float thr0 = thr_sh;
#pragma unroll
        for (int k = 0; k < kPerThread; k++) {
            const uint64_t i = i0 + k;
            if (i <= last) {
                const float l = d[i - 1], v = d[i], r = d[i + 1];
                const bool pk = use_max ? (v > l && v > r && v > thr0)
                                        : (v < l && v < r && v < thr0);
                flags |= (pk ? 1u : 0u) << k;
            }
        }
        // (2) order-preserving compaction: exclusive scan of popcounts.
        const uint32_t mine = __popc(flags);
        uint32_t incl = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) warp_tot[wid] = incl;
        __syncthreads();
        if (tid == 0) {
            uint32_t run = 0;
            for (int w = 0; w < kPeakThreads / 32; w++) {
                const uint32_t t = warp_tot[w];
                warp_tot[w] = run;
                run += t;
            }
            chunk_count = run;
        }
        __syncthreads();
        uint32_t pos = warp_tot[wid] + incl - mine;
#pragma unroll
        for (int k = 0; k < kPerThread; k++) {
            if (flags & (1u << k)) {
                ext_idx[pos] = (int64_t)(i0 + k);
                ext_val[pos] = d[i0 + k];
                pos++;
            }
        }
        __syncthreads();
        // (3) replay.  Up to 32 peaks: warp 0, 32 extrema at a time; lanes
        // whose extremum no longer beats the threshold are dropped by one
        // ballot (the threshold only gets stricter), the rest are fed in
        // index order.
        if (warp_list) {
            if (wid == 0) {
                warp_replay(w, lane, ext_idx, ext_val, chunk_count, md, use_max);
                if (lane == 0) thr_sh = w.thr;
            }
        } else if (tid == 0) {
            // More than 32 peaks: one thread, the list in shared memory.
            const uint32_t ne = chunk_count;
            for (uint32_t e = 0; e < ne; e++) {
                const int64_t i = ext_idx[e];
                const float v = ext_val[e];
                // Promotion that happened strictly before index i.
                if (s.has_cand && (uint64_t)s.cand_idx + (md > 0 ? md - 1 : 0) < (uint64_t)i)
                    promote(s);
                // feed(i): peak test against the current threshold.
                if (better(use_max, v, s.thr) &&
                    (!s.has_cand || better(use_max, v, s.cand_val))) {
                    s.cand_idx = i;
                    s.cand_val = v;
                    s.has_cand = true;
                }
                // Distance after feeding i: i - cand_idx + 1.
                if (s.has_cand && (uint64_t)(i - s.cand_idx) + 1 >= md) promote(s);
            }
            thr_sh = s.thr;
        }
        __syncthreads();
    }
    // Finalize (peaks.rs:207-209) and write the row.
    if (warp_list) {
        if (wid == 0) {
            warp_promote(w, lane);
            if (lane < (int)n_peaks) {
                const bool have = (uint32_t)lane < w.count;
                out_idx[c * n_peaks + lane] = have ? w.idx : -1;
                out_val[c * n_peaks + lane] = have ? w.val : 0.0f;
            }
        }
        return;
    }
    if (tid == 0) promote(s);
    __syncthreads();
    const uint32_t count = __shfl_sync(0xffffffffu, s.count, 0);
    if (wid == 0) {
        for (uint32_t k = lane; k < n_peaks; k += 32) {
            const bool have = k < count;
            out_idx[c * n_peaks + k] = have ? top_idx[k] : -1;
            out_val[c * n_peaks + k] = have ? top_val[k] : 0.0f;
        }
    }
}


// Top lists of at most 32 peaks: a warp per row, no CTA barrier, so up to 64
// rows per SM replay their extrema at once (the CTA-per-row kernel above
// runs one replaying warp per 256 threads while the rest wait at its
// barriers).  A warp takes 256 samples per step: lane l tests samples
// base + 32 k + l (k < 8; coalesced loads, neighbours from the same
// lines), the extrema that beat the current threshold are compacted in
// index order by ballot into the warp's shared buffer, then replayed.
constexpr int kRowWarps = 4;
constexpr uint32_t kWarpStep = 256;

__global__ void __launch_bounds__(kRowWarps * 32, 10)
    peaks_warp_kernel(const float* __restrict__ pg, uint64_t n_rows, uint64_t flat_len,
                      uint32_t n_peaks, uint32_t min_distance, int use_max_i,
                      int64_t* __restrict__ out_idx, float* __restrict__ out_val) {
    __shared__ int64_t s_idx[kRowWarps][kWarpStep];
    __shared__ float s_val[kRowWarps][kWarpStep];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint64_t c = (uint64_t)blockIdx.x * kRowWarps + wid;
    if (c >= n_rows) return;  // the whole warp; no CTA-wide barrier follows
    const float* d = pg + c * flat_len;
    const bool use_max = use_max_i != 0;
    int64_t* ext_idx = s_idx[wid];
    float* ext_val = s_val[wid];

    WarpTop w;
    w.idx = -1;
    w.val = 0.0f;
    w.count = 0;
    w.n_peaks = n_peaks;
    w.use_max = use_max;
    w.has_cand = false;
    w.cand_idx = -1;
    w.cand_val = use_max ? -INFINITY : INFINITY;
    w.thr = use_max ? -INFINITY : INFINITY;
    const uint64_t md = min_distance;
    const unsigned lt_mask = (1u << lane) - 1u;

    const uint64_t last = (flat_len >= 2) ? flat_len - 2 : 0;
    for (uint64_t base = 1; flat_len >= 3 && base <= last; base += kWarpStep) {
        const float thr0 = w.thr;  // uniform across the warp
        float v[8];
        bool pk[8];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const uint64_t i = base + (uint64_t)k * 32 + lane;
            pk[k] = false;
            v[k] = 0.0f;
            if (i <= last) {
                const float l = d[i - 1], x = d[i], r = d[i + 1];
                v[k] = x;
                pk[k] = use_max ? (x > l && x > r && x > thr0) : (x < l && x < r && x < thr0);
            }
        }
        uint32_t ne = 0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            const unsigned m = __ballot_sync(0xffffffffu, pk[k]);
            if (pk[k]) {
                const uint32_t pos = ne + __popc(m & lt_mask);
                ext_idx[pos] = (int64_t)(base + (uint64_t)k * 32 + lane);
                ext_val[pos] = v[k];
            }
            ne += __popc(m);
        }
        __syncwarp();
        warp_replay(w, lane, ext_idx, ext_val, ne, md, use_max);
        __syncwarp();
    }
    warp_promote(w, lane);
    if (lane < (int)n_peaks) {
        const bool have = (uint32_t)lane < w.count;
        out_idx[c * n_peaks + lane] = have ? w.idx : -1;
        out_val[c * n_peaks + lane] = have ? w.val : 0.0f;
    }
}

}  // namespace

cudaError_t launch_peaks(const float* pg, uint64_t n_curves, uint64_t flat_len,
                         uint32_t n_peaks, uint32_t min_distance, int use_max,
                         int64_t* out_idx, float* out_val, cudaStream_t stream) {
    if (n_curves == 0 || n_peaks == 0) return cudaSuccess;
    if (n_peaks <= 32) {
        const uint64_t blocks = (n_curves + kRowWarps - 1) / kRowWarps;
        if (blocks > 0x7FFFFFFFull) return cudaErrorInvalidValue;
        peaks_warp_kernel<<<(unsigned)blocks, kRowWarps * 32, 0, stream>>>(
            pg, n_curves, flat_len, n_peaks, min_distance, use_max, out_idx, out_val);
        return cudaGetLastError();
    }
    const size_t smem = (size_t)kChunk * 12 + (size_t)n_peaks * 12;
    if (smem > 227u * 1024u) return cudaErrorInvalidValue;  // n_peaks > ~18000
    cudaError_t e = cudaFuncSetAttribute(peaks_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    peaks_kernel<<<(unsigned)n_curves, kPeakThreads, smem, stream>>>(
        pg, flat_len, n_peaks, min_distance, use_max, out_idx, out_val);
    return cudaGetLastError();
}

}  // namespace pfk
