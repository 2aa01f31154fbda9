// pf_stats.cu -- the 'stats' output on the device: per periodogram row, the
// values the reference computes on the host with numpy
// (periodfind/__init__.py:338-400, Statistics.statistics_from_data):
//   mean   = np.mean(data), std = np.std(data)   (float32, numpy's pairwise
//            summation order: leaves of <= 128 elements summed with eight
//            accumulators, halves split at multiples of 8, as np.add.reduce)
//   median = np.median(data), mad = np.median(|data - median|)
//            (exact order statistics; the mean of the two middle values for
//            an even count; NaN anywhere gives NaN, as numpy)
//   the n best entries (smallest for CE, largest otherwise; NaN ranks
//            largest, as np.argpartition), best first.
// One CTA per curve; order statistics by 8-bit radix selection over
// order-preserving keys, reading the row from global memory (L2).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "pf_launch.h"

namespace pfk {

namespace {

constexpr int kStatThreads = 256;
constexpr int kLeaf = 128;  // numpy's pairwise block size

// Order-preserving key of a float (NaN ranks above +inf, as in numpy sorts).
__device__ __forceinline__ uint32_t fkey(float v) {
    if (isnan(v)) return 0xFFFFFFFFu;
    const uint32_t b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unkey(uint32_t k) {
    if (k == 0xFFFFFFFFu) return __uint_as_float(0x7FC00000u);
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

// The element transform of each pass: the row itself, its squared deviation
// from the mean (np.std), or its absolute deviation from the median (MAD).
enum : int { T_X = 0, T_SQDEV = 1, T_ABSDEV = 2 };
__device__ __forceinline__ float elem(const float* x, uint32_t i, int tr, float ref) {
    const float v = x[i];
    if (tr == T_SQDEV) {
        const float d = __fsub_rn(v, ref);
        return __fmul_rn(d, d);
    }
    if (tr == T_ABSDEV) return fabsf(__fsub_rn(v, ref));
    return v;
}

// numpy's pairwise_sum on one leaf (n <= 128), IEEE float32 operations.
__device__ float leaf_sum(const float* x, uint32_t lo, uint32_t n, int tr, float ref) {
    if (n < 8) {
        float res = -0.0f;
        for (uint32_t i = 0; i < n; i++) res = __fadd_rn(res, elem(x, lo + i, tr, ref));
        return res;
    }
    float r[8];
#pragma unroll
    for (int k = 0; k < 8; k++) r[k] = elem(x, lo + k, tr, ref);
    uint32_t i = 8;
    for (; i < n - (n % 8); i += 8) {
#pragma unroll
        for (int k = 0; k < 8; k++) r[k] = __fadd_rn(r[k], elem(x, lo + i + k, tr, ref));
    }
    float res = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                          __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
    for (; i < n; i++) res = __fadd_rn(res, elem(x, lo + i, tr, ref));
    return res;
}

// The leaves of numpy's recursion over [lo, lo + n), left to right: a range
// above kLeaf splits at n2 = (n / 2) rounded down to a multiple of 8.
__device__ void list_leaves(uint32_t lo, uint32_t n, uint32_t* lo_out, uint32_t* len_out,
                            uint32_t& count) {
    if (n <= (uint32_t)kLeaf) {
        lo_out[count] = lo;
        len_out[count] = n;
        count++;
        return;
    }
    uint32_t n2 = n / 2;
    n2 -= n2 % 8;
    list_leaves(lo, n2, lo_out, len_out, count);
    list_leaves(lo + n2, n - n2, lo_out, len_out, count);
}

// The leaf sums combined in numpy's recursion order: pairwise_sum(left) +
// pairwise_sum(right) at every split.
__device__ float combine_leaves(uint32_t n, const float* leaf, uint32_t& next) {
    if (n <= (uint32_t)kLeaf) return leaf[next++];
    uint32_t n2 = n / 2;
    n2 -= n2 % 8;
    const float a = combine_leaves(n2, leaf, next);
    const float b = combine_leaves(n - n2, leaf, next);
    return __fadd_rn(a, b);
}

// np.add.reduce of the transformed row, all threads participating.
__device__ float pairwise_row(const float* x, uint32_t n, int tr, float ref, uint32_t n_leaves,
                             const uint32_t* leaf_lo, const uint32_t* leaf_len, float* leaf) {
    for (uint32_t l = threadIdx.x; l < n_leaves; l += kStatThreads)
        leaf[l] = leaf_sum(x, leaf_lo[l], leaf_len[l], tr, ref);
    __syncthreads();
    __shared__ float result;
    if (threadIdx.x == 0) {
        uint32_t next = 0;
        result = combine_leaves(n, leaf, next);
    }
    __syncthreads();
    const float r = result;
    __syncthreads();
    return r;
}

// Key of the k-th smallest transformed element (0-based), by four 8-bit
// radix passes over the row.  All threads participate.
__device__ uint32_t select_key(const float* x, uint32_t n, int tr, float ref, uint32_t k,
                               uint32_t* hist) {
    __shared__ uint32_t s_prefix, s_k;
    if (threadIdx.x == 0) {
        s_prefix = 0;
        s_k = k;
    }
    for (int pass = 0; pass < 4; pass++) {
        const int shift = 24 - 8 * pass;
        for (int b = threadIdx.x; b < 256; b += kStatThreads) hist[b] = 0;
        __syncthreads();
        const uint32_t prefix = s_prefix;
        const uint32_t mask = pass == 0 ? 0u : (0xFFFFFFFFu << (32 - 8 * pass));
        for (uint32_t i = threadIdx.x; i < n; i += kStatThreads) {
            const uint32_t key = fkey(elem(x, i, tr, ref));
            if ((key & mask) == prefix) atomicAdd(&hist[(key >> shift) & 0xFFu], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t rem = s_k;
            int b = 0;
            for (; b < 255 && rem >= hist[b]; b++) rem -= hist[b];
            s_prefix = prefix | ((uint32_t)b << shift);
            s_k = rem;
        }
        __syncthreads();
    }
    const uint32_t key = s_prefix;
    __syncthreads();
    return key;
}

// Count of transformed elements with key <= `key`, and the smallest key
// above it (0xFFFFFFFF if none).  All threads participate.
__device__ void count_and_next(const float* x, uint32_t n, int tr, float ref, uint32_t key,
                               uint32_t* le, uint32_t* next) {
    __shared__ uint32_t s_le, s_next;
    if (threadIdx.x == 0) {
        s_le = 0;
        s_next = 0xFFFFFFFFu;
    }
    __syncthreads();
    uint32_t c = 0, nx = 0xFFFFFFFFu;
    for (uint32_t i = threadIdx.x; i < n; i += kStatThreads) {
        const uint32_t kk = fkey(elem(x, i, tr, ref));
        if (kk <= key) c++;
        else nx = min(nx, kk);
    }
    atomicAdd(&s_le, c);
    atomicMin(&s_next, nx);
    __syncthreads();
    *le = s_le;
    *next = s_next;
    __syncthreads();
}

// np.median of the transformed row (NaN if any element is NaN).
__device__ float median_row(const float* x, uint32_t n, int tr, float ref, bool any_nan,
                            uint32_t* hist) {
    if (any_nan) return __uint_as_float(0x7FC00000u);
    const uint32_t k1 = (n - 1) / 2;
    const uint32_t a = select_key(x, n, tr, ref, k1, hist);
    if (n % 2) return unkey(a);
    uint32_t le, nx;
    count_and_next(x, n, tr, ref, a, &le, &nx);
    const uint32_t b = (le >= k1 + 2) ? a : nx;
    // the mean of the two middle values: np.mean of a two-element array
    return __fdiv_rn(__fadd_rn(__fadd_rn(-0.0f, unkey(a)), unkey(b)), 2.0f);
}

// Rows of at most kSortMax cells are sorted once in shared memory instead of
// radix-selected pass by pass: the median, the MAD and the best entries are
// then read off the sorted row.
constexpr uint32_t kSortMax = 8192;

__host__ __device__ inline uint32_t sort_width(uint32_t n) {
    uint32_t p = 1;
    while (p < n) p <<= 1;
    return p;
}

// Dynamic shared memory of stats_kernel: the leaf table, then (sorted path)
// the row and its sort records.
__host__ __device__ inline size_t stats_rowcopy_offset(uint32_t leaf_cap) {
    return ((size_t)leaf_cap * 12 + 15) & ~(size_t)15;
}
__host__ __device__ inline size_t stats_sortrec_offset(uint32_t leaf_cap, uint32_t n) {
    return stats_rowcopy_offset(leaf_cap) + (((size_t)n * 4 + 15) & ~(size_t)15);
}

// Ascending bitonic sort of w (a power of two) 64-bit records, all threads.
__device__ void bitonic_sort(unsigned long long* s, uint32_t w) {
    for (uint32_t k = 2; k <= w; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < w; i += kStatThreads) {
                const uint32_t p = i ^ j;
                if (p > i) {
                    const unsigned long long a = s[i], b = s[p];
                    const bool up = (i & k) == 0;
                    if ((a > b) == up) {
                        s[i] = b;
                        s[p] = a;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// The k-th smallest (0-based) of the merge of two non-decreasing sequences
// A (na values) and B (nb values), k < na + nb: binary search for how many
// of the k + 1 smallest come from A.
template <class FA, class FB>
__device__ float kth_of_merge(FA A, uint32_t na, FB B, uint32_t nb, uint32_t k) {
    uint32_t lo = (k + 1 > nb) ? k + 1 - nb : 0u;
    uint32_t hi = min(na, k + 1);
    while (lo < hi) {
        const uint32_t i = (lo + hi) / 2;
        const uint32_t j = k + 1 - i;
        if (i < na && j > 0 && B(j - 1) > A(i)) lo = i + 1;
        else hi = i;
    }
    const uint32_t i = lo, j = k + 1 - lo;
    if (i == 0) return B(j - 1);
    if (j == 0) return A(i - 1);
    return fmaxf(A(i - 1), B(j - 1));
}

__global__ void __launch_bounds__(kStatThreads)
    stats_kernel(const float* __restrict__ pg, uint32_t n, int use_max, uint32_t n_top,
                 uint32_t leaf_cap, float* __restrict__ stats, int64_t* __restrict__ top_idx,
                 float* __restrict__ top_val) {
    extern __shared__ __align__(16) unsigned char ssm[];
    uint32_t* leaf_lo = reinterpret_cast<uint32_t*>(ssm);
    uint32_t* leaf_len = leaf_lo + leaf_cap;
    float* leaf = reinterpret_cast<float*>(leaf_len + leaf_cap);
    __shared__ uint32_t hist[256];
    __shared__ uint32_t s_leaves;
    __shared__ int s_nan;
    const uint64_t c = blockIdx.x;
    const float* x = pg + c * (uint64_t)n;

    if (threadIdx.x == 0) {
        uint32_t count = 0;
        list_leaves(0, n, leaf_lo, leaf_len, count);  // leaf_cap leaves (host count)
        s_leaves = count;
        s_nan = 0;
    }
    __syncthreads();
    const uint32_t n_leaves = s_leaves;  // == leaf_cap (the same recursion on the host)
    const bool sorted = n <= kSortMax;
    unsigned long long* rec = nullptr;
    const uint32_t w = sort_width(n);
    int nan_local = 0;
    if (sorted) {
        // The row into shared memory, and one sort record per cell: the
        // cell's order key (complemented when the largest is best, so that
        // an ascending sort puts the best first) above its index, so equal
        // values keep the lowest index first.  Padding sorts last.
        float* xs = reinterpret_cast<float*>(ssm + stats_rowcopy_offset(leaf_cap));
        rec = reinterpret_cast<unsigned long long*>(ssm + stats_sortrec_offset(leaf_cap, n));
        for (uint32_t i = threadIdx.x; i < w; i += kStatThreads) {
            if (i < n) {
                const float v = x[i];
                xs[i] = v;
                nan_local |= isnan(v) ? 1 : 0;
                const uint32_t k = use_max ? ~fkey(v) : fkey(v);
                rec[i] = ((unsigned long long)k << 32) | i;
            } else {
                rec[i] = ~0ull;
            }
        }
        x = xs;
    } else {
        for (uint32_t i = threadIdx.x; i < n; i += kStatThreads) nan_local |= isnan(x[i]) ? 1 : 0;
    }
    if (nan_local) atomicOr(&s_nan, 1);
    __syncthreads();

    // np.mean, then np.std as in numpy's _var: mean kept as float32, the
    // squared deviations summed pairwise, divided by n, square root.
    const float fn = (float)n;
    const float sum = pairwise_row(x, n, T_X, 0.0f, n_leaves, leaf_lo, leaf_len, leaf);
    const float mean = __fdiv_rn(sum, fn);
    const float ssq = pairwise_row(x, n, T_SQDEV, mean, n_leaves, leaf_lo, leaf_len, leaf);
    const float stdv = __fsqrt_rn(__fdiv_rn(ssq, fn));
    const bool any_nan = s_nan != 0;
    if (sorted) {
        bitonic_sort(rec, w);
        // Values in ascending order: rec holds them best first.
        auto asc = [&](uint32_t pos) -> float {
            const uint32_t k = (uint32_t)(rec[use_max ? n - 1 - pos : pos] >> 32);
            return unkey(use_max ? ~k : k);
        };
        if (threadIdx.x == 0) {
            float med = __uint_as_float(0x7FC00000u), mad = med;
            if (!any_nan && n > 0) {
                // np.median: the middle value, or the mean of the two
                // middle values (np.mean of a two-element array).
                const uint32_t k1 = (n - 1) / 2;
                med = (n % 2) ? asc(k1)
                              : __fdiv_rn(__fadd_rn(__fadd_rn(-0.0f, asc(k1)), asc(k1 + 1)),
                                          2.0f);
                // MAD: the deviations |v - med| of the values below the
                // median, taken downwards, and of the rest, taken upwards,
                // are two non-decreasing sequences (rounding is monotone);
                // their merged order statistics give np.median of |x - med|.
                uint32_t lo = 0, hi = n;  // la = number of values below med
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) / 2;
                    if (asc(mid) < med) lo = mid + 1;
                    else hi = mid;
                }
                const uint32_t la = lo;
                auto A = [&](uint32_t i) { return fabsf(__fsub_rn(asc(la - 1 - i), med)); };
                auto B = [&](uint32_t j) { return fabsf(__fsub_rn(asc(la + j), med)); };
                const float d1 = kth_of_merge(A, la, B, n - la, k1);
                mad = (n % 2) ? d1
                              : __fdiv_rn(__fadd_rn(__fadd_rn(-0.0f, d1),
                                                    kth_of_merge(A, la, B, n - la, k1 + 1)),
                                          2.0f);
            }
            stats[4 * c + 0] = mean;
            stats[4 * c + 1] = stdv;
            stats[4 * c + 2] = med;
            stats[4 * c + 3] = mad;
        }
        // The n_top best: the first records, best first, lowest index
        // first among equal values; -1 / 0 beyond the row.
        for (uint32_t a = threadIdx.x; a < n_top; a += kStatThreads) {
            if (a < n) {
                const uint32_t i = (uint32_t)rec[a];
                top_idx[c * n_top + a] = i;
                top_val[c * n_top + a] = x[i];
            } else {
                top_idx[c * n_top + a] = -1;
                top_val[c * n_top + a] = 0.0f;
            }
        }
        return;
    }
    const float med = median_row(x, n, T_X, 0.0f, any_nan, hist);
    const float mad = median_row(x, n, T_ABSDEV, med, any_nan, hist);
    if (threadIdx.x == 0) {
        stats[4 * c + 0] = mean;
        stats[4 * c + 1] = stdv;
        stats[4 * c + 2] = med;
        stats[4 * c + 3] = mad;
    }

    // The n_top best: keys of the n_top-th best as a threshold, then the
    // entries strictly better plus the lowest-index ties, best first.
    if (n_top == 0) return;
    const uint32_t m = min(n_top, n);
    const uint32_t kth = use_max ? n - m : m - 1;
    const uint32_t thr = select_key(x, n, T_X, 0.0f, kth, hist);
    __shared__ uint32_t s_cnt;
    if (threadIdx.x == 0) s_cnt = 0;
    __syncthreads();
    // Strictly better entries first (there are fewer than m of them).
    for (uint32_t i = threadIdx.x; i < n; i += kStatThreads) {
        const uint32_t kk = fkey(x[i]);
        if (use_max ? kk > thr : kk < thr) {
            const uint32_t slot = atomicAdd(&s_cnt, 1u);
            top_idx[c * n_top + slot] = i;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // Ties at the threshold, lowest indices first, up to m in total.
        uint32_t cnt = s_cnt;
        for (uint32_t i = 0; i < n && cnt < m; i++)
            if (fkey(x[i]) == thr) top_idx[c * n_top + cnt++] = i;
        // Best first (insertion sort on (key, index); m is small).
        int64_t* ti = top_idx + c * n_top;
        for (uint32_t a = 1; a < m; a++) {
            const int64_t v = ti[a];
            const uint32_t kv = fkey(x[v]);
            int b = (int)a - 1;
            while (b >= 0) {
                const uint32_t kb = fkey(x[ti[b]]);
                const bool after = use_max ? (kb < kv || (kb == kv && ti[b] > v))
                                           : (kb > kv || (kb == kv && ti[b] > v));
                if (!after) break;
                ti[b + 1] = ti[b];
                b--;
            }
            ti[b + 1] = v;
        }
        for (uint32_t a = 0; a < n_top; a++) {
            if (a < m) {
                top_val[c * n_top + a] = x[ti[a]];
            } else {
                ti[a] = -1;
                top_val[c * n_top + a] = 0.0f;
            }
        }
    }
}

// Magnitude preparation on the device, a CTA per curve, with the values
// the reference's prepare_magnitudes gets from numpy (periodfind/_utils.py:
// 29-45): kind 1 centres, m - np.mean(m) (numpy's pairwise float32 sum
// divided by n); kind 2 normalises, ((m - min) / (max - min)) * 0.999 +
// 5e-4 in float32 with NaN propagating through min / max.  Curve c is
// m[off[c] .. off[c+1]); its output goes to the same place in out.
__global__ void __launch_bounds__(kStatThreads)
    prep_mags_kernel(const float* __restrict__ m, const int64_t* __restrict__ off, int kind,
                     uint32_t leaf_cap, float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char psm[];
    __shared__ uint32_t s_leaves;
    __shared__ float s_lo[kStatThreads / 32], s_hi[kStatThreads / 32];
    __shared__ int s_nan;
    const uint64_t c = blockIdx.x;
    const int64_t lo = off[c];
    const uint32_t n = (uint32_t)(off[c + 1] - lo);
    if (n == 0) return;  // uniform over the CTA
    const float* x = m + lo;
    float* y = out + lo;
    if (kind == 1) {
        // leaf arrays for leaf_cap leaves: the host's maximum over the curves
        uint32_t* leaf_lo = reinterpret_cast<uint32_t*>(psm);
        uint32_t* leaf_len = leaf_lo + leaf_cap;
        float* leaf = reinterpret_cast<float*>(leaf_len + leaf_cap);
        if (threadIdx.x == 0) {
            uint32_t count = 0;
            list_leaves(0, n, leaf_lo, leaf_len, count);
            s_leaves = count;
        }
        __syncthreads();
        const float sum = pairwise_row(x, n, T_X, 0.0f, s_leaves, leaf_lo, leaf_len, leaf);
        const float mean = __fdiv_rn(sum, (float)n);
        for (uint32_t i = threadIdx.x; i < n; i += kStatThreads) y[i] = __fsub_rn(x[i], mean);
        return;
    }
    // np.min / np.max: exact, any order; NaN anywhere gives NaN.
    float mn = INFINITY, mx = -INFINITY;
    int nan_local = 0;
    for (uint32_t i = threadIdx.x; i < n; i += kStatThreads) {
        const float v = x[i];
        nan_local |= isnan(v) ? 1 : 0;
        mn = fminf(mn, v);
        mx = fmaxf(mx, v);
    }
    if (threadIdx.x == 0) s_nan = 0;
    __syncthreads();
    if (nan_local) atomicOr(&s_nan, 1);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    if ((threadIdx.x & 31) == 0) {
        s_lo[threadIdx.x >> 5] = mn;
        s_hi[threadIdx.x >> 5] = mx;
    }
    __syncthreads();
    float cmin = s_lo[0], cmax = s_hi[0];
    for (int w = 1; w < kStatThreads / 32; w++) {
        cmin = fminf(cmin, s_lo[w]);
        cmax = fmaxf(cmax, s_hi[w]);
    }
    if (s_nan) cmin = cmax = __uint_as_float(0x7FC00000u);
    const float range = __fsub_rn(cmax, cmin);
    for (uint32_t i = threadIdx.x; i < n; i += kStatThreads)
        y[i] = __fadd_rn(__fmul_rn(__fdiv_rn(__fsub_rn(x[i], cmin), range), 0.999f), 5e-4f);
}

}  // namespace

uint32_t stats_leaf_count(uint32_t n) {
    // The number of leaves of numpy's recursion over n elements (host side).
    uint32_t count = 0;
    uint32_t stack[64];
    int sp = 0;
    stack[sp++] = n;
    while (sp > 0) {
        const uint32_t m = stack[--sp];
        if (m <= (uint32_t)kLeaf) {
            count++;
            continue;
        }
        uint32_t n2 = m / 2;
        n2 -= n2 % 8;
        stack[sp++] = m - n2;
        stack[sp++] = n2;
    }
    return count;
}

cudaError_t launch_stats(const float* pg, uint64_t n_curves, uint32_t n_cells, int use_max,
                         uint32_t n_top, float* stats, int64_t* top_idx, float* top_val,
                         cudaStream_t s) {
    if (n_curves == 0) return cudaSuccess;
    const uint32_t leaves = n_cells ? stats_leaf_count(n_cells) : 1;
    size_t smem = (size_t)leaves * 12;
    if (n_cells <= kSortMax)
        smem = stats_sortrec_offset(leaves, n_cells) + (size_t)sort_width(n_cells) * 8;
    if (smem > 200u * 1024u) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(stats_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    stats_kernel<<<(unsigned)n_curves, kStatThreads, smem, s>>>(pg, n_cells, use_max, n_top,
                                                                leaves, stats, top_idx, top_val);
    return cudaGetLastError();
}

cudaError_t launch_prep_mags(const float* m, const int64_t* d_off, uint64_t n_curves,
                             uint32_t leaf_cap, int kind, float* out, cudaStream_t s) {
    if (n_curves == 0) return cudaSuccess;
    if (kind != 1 && kind != 2) return cudaErrorInvalidValue;
    if (n_curves > 0x7FFFFFFFull) return cudaErrorInvalidValue;
    const uint32_t leaves = leaf_cap ? leaf_cap : 1;
    const size_t smem = (size_t)leaves * 12;
    if (smem > 200u * 1024u) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(prep_mags_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    prep_mags_kernel<<<(unsigned)n_curves, kStatThreads, smem, s>>>(m, d_off, kind, leaves,
                                                                     out);
    return cudaGetLastError();
}

}  // namespace pfk
