// pf_prep.cu -- per-curve preparation that the reference does on the host.
//
//  - AOV mean: the reference computes it on the host, per curve, with a
//    sequential f32 sum and an IEEE divide (ArrayMean, periodfind/cuda/
//    aov.cu:251-259; rust/src/aov.rs:27).  Reproduced here in the same order.
//  - AOV fixed-point magnitudes for the exact accumulator (AOVACC_FIX).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "pf_launch.h"
#include "pf_types.h"

namespace pfk {

namespace {

constexpr int kPrepThreads = 256;
constexpr uint32_t kChunk = 4096;

// One CTA per curve: the CTA stages the magnitudes through shared memory
// and one thread adds them in point order.
__global__ void __launch_bounds__(kPrepThreads)
    aov_mean_kernel(const float* __restrict__ m, CurveDesc* __restrict__ curves,
                    uint32_t n_curves) {
    __shared__ float chunk[kChunk];
    const uint32_t c = blockIdx.x;
    if (c >= n_curves) return;
    const CurveDesc cd = curves[c];
    float sum = 0.0f;
    for (uint32_t base = 0; base < cd.n; base += kChunk) {
        const uint32_t cnt = min(kChunk, cd.n - base);
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < cnt; i += kPrepThreads) chunk[i] = m[cd.off + base + i];
        __syncthreads();
        if (threadIdx.x == 0) {
            for (uint32_t i = 0; i < cnt; i++) sum = __fadd_rn(sum, chunk[i]);
        }
    }
    if (threadIdx.x == 0) curves[c].avg = __fdiv_rn(sum, (float)cd.n);
}

template <typename T, typename Op>
__device__ T block_reduce(T v, T* scratch, Op op) {
    // Fixed-order tree: deterministic for a given block size.
    scratch[threadIdx.x] = v;
    __syncthreads();
    for (int s = kPrepThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) scratch[threadIdx.x] = op(scratch[threadIdx.x], scratch[threadIdx.x + s]);
        __syncthreads();
    }
    T r = scratch[0];
    __syncthreads();
    return r;
}

// Fixed-point magnitudes: q = rint((m - min) * scale) with scale chosen so
// that a bin's sum of up to n * overlap values stays below 2^44, leaving the
// top 20 bits of a u64 for the bin count: aux64 = (1 << 44) + q.
__global__ void __launch_bounds__(kPrepThreads)
    aov_fix_kernel(const float* __restrict__ m, uint64_t* __restrict__ aux64,
                   CurveDesc* __restrict__ curves, uint32_t n_curves, uint32_t overlap) {
    __shared__ double dscr[kPrepThreads];
    __shared__ float fscr[kPrepThreads];
    __shared__ unsigned long long uscr[kPrepThreads];
    const uint32_t c = blockIdx.x;
    if (c >= n_curves) return;
    const CurveDesc cd = curves[c];
    const float* mc = m + cd.off;

    float mn = __int_as_float(0x7f800000), mx = -__int_as_float(0x7f800000);
    for (uint32_t i = threadIdx.x; i < cd.n; i += kPrepThreads) {
        mn = fminf(mn, mc[i]);
        mx = fmaxf(mx, mc[i]);
    }
    mn = block_reduce(mn, fscr, [](float a, float b) { return fminf(a, b); });
    mx = block_reduce(mx, fscr, [](float a, float b) { return fmaxf(a, b); });

    // Bits needed for a bin total: ceil(log2(n * overlap + 1)).
    const unsigned long long tot = (unsigned long long)cd.n * overlap + 1ull;
    const int need = 64 - __clzll(tot - 1ull);
    const int kbits = max(1, kFixCountShift - need);
    const double span = (double)mx - (double)mn;
    const double scale = (span > 0.0) ? (double)((1ull << kbits) - 1ull) / span : 0.0;

    unsigned long long sx = 0ull;
    double sx2 = 0.0;
    const uint32_t n4 = (cd.n + 3u) & ~3u;
    for (uint32_t i = threadIdx.x; i < n4; i += kPrepThreads) {
        uint64_t v = 0ull;
        if (i < cd.n) {
            const double x = rint(((double)mc[i] - (double)mn) * scale);
            const unsigned long long q = (unsigned long long)x;
            sx += q;
            sx2 = __fma_rn((double)q, (double)q, sx2);
            v = (1ull << kFixCountShift) + q;
        }
        aux64[cd.off + i] = v;
    }
    sx = block_reduce(sx, uscr, [](unsigned long long a, unsigned long long b) { return a + b; });
    sx2 = block_reduce(sx2, dscr, [](double a, double b) { return a + b; });
    if (threadIdx.x == 0) {
        curves[c].fix_mn = (double)mn;
        curves[c].fix_scale = scale;
        curves[c].fix_sumx = (double)sx;
        curves[c].fix_sumx2 = sx2;
    }
}

// Gather caller-packed device curves into the library's layout (16-byte
// aligned starts, zero padding to a multiple of 4 points).
__global__ void __launch_bounds__(kPrepThreads)
    pack_kernel(const float* __restrict__ src_t, const float* __restrict__ src_m,
                const int64_t* __restrict__ src_off, const CurveDesc* __restrict__ curves,
                uint32_t n_curves, float* __restrict__ dst_t, float* __restrict__ dst_m) {
    const uint32_t c = blockIdx.x;
    if (c >= n_curves) return;
    const CurveDesc cd = curves[c];
    const int64_t so = src_off[c];
    const uint32_t n4 = (cd.n + 3u) & ~3u;
    for (uint32_t i = threadIdx.x; i < n4; i += kPrepThreads) {
        const bool in = i < cd.n;
        dst_t[cd.off + i] = in ? src_t[so + i] : 0.0f;
        dst_m[cd.off + i] = in ? src_m[so + i] : 0.0f;
    }
}

// max |t| over the packed batch (padding is zero).  |t| as float bits is
// monotone in the value, so an unsigned max is a float max.
__global__ void tmax_kernel(const float* __restrict__ t, size_t n, unsigned* __restrict__ out) {
    unsigned mx = 0u;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        mx = max(mx, __float_as_uint(fabsf(t[i])));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

// 32-bit fixed-point magnitudes for the bin kernel: k = min(24, 32 -
// ceil(log2(n + 1))) bits so a bin's sum of up to n values fits in 32 bits.
__global__ void __launch_bounds__(kPrepThreads)
    aov_fix32_kernel(const float* __restrict__ m, uint32_t* __restrict__ aux32,
                     CurveDesc* __restrict__ curves, uint32_t n_curves) {
    __shared__ double dscr[kPrepThreads];
    __shared__ float fscr[kPrepThreads];
    __shared__ unsigned long long uscr[kPrepThreads];
    const uint32_t c = blockIdx.x;
    if (c >= n_curves) return;
    const CurveDesc cd = curves[c];
    const float* mc = m + cd.off;
    float mn = __int_as_float(0x7f800000), mx = -__int_as_float(0x7f800000);
    for (uint32_t i = threadIdx.x; i < cd.n; i += kPrepThreads) {
        mn = fminf(mn, mc[i]);
        mx = fmaxf(mx, mc[i]);
    }
    mn = block_reduce(mn, fscr, [](float a, float b) { return fminf(a, b); });
    mx = block_reduce(mx, fscr, [](float a, float b) { return fmaxf(a, b); });
    const unsigned long long tot = (unsigned long long)cd.n + 1ull;
    const int need = 64 - __clzll(tot - 1ull);
    const int kbits = min(24, 32 - need);
    const double span = (double)mx - (double)mn;
    const double scale = (span > 0.0 && kbits > 0) ? (double)((1u << kbits) - 1u) / span : 0.0;
    unsigned long long sx = 0ull;
    double sx2 = 0.0;
    const uint32_t n4 = (cd.n + 3u) & ~3u;
    for (uint32_t i = threadIdx.x; i < n4; i += kPrepThreads) {
        uint32_t v = 0u;
        if (i < cd.n) {
            v = (uint32_t)rint(((double)mc[i] - (double)mn) * scale);
            sx += v;
            sx2 = __fma_rn((double)v, (double)v, sx2);
        }
        aux32[cd.off + i] = v;
    }
    sx = block_reduce(sx, uscr, [](unsigned long long a, unsigned long long b) { return a + b; });
    sx2 = block_reduce(sx2, dscr, [](double a, double b) { return a + b; });
    if (threadIdx.x == 0) {
        curves[c].fix_mn = (double)mn;
        curves[c].fix_scale = scale;
        curves[c].fix_sumx = (double)sx;
        curves[c].fix_sumx2 = sx2;
    }
}

}  // namespace

cudaError_t launch_tmax(const float* t, size_t n, unsigned* tmax_bits, cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(tmax_bits, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess || n == 0) return e;
    const int blocks = (int)std::min<size_t>((n + 255) / 256, 1184);
    tmax_kernel<<<blocks, 256, 0, stream>>>(t, n, tmax_bits);
    return cudaGetLastError();
}

cudaError_t launch_aov_fix32_prep(const float* m, uint32_t* aux32, CurveDesc* curves,
                                  uint32_t n_curves, cudaStream_t stream) {
    if (n_curves == 0) return cudaSuccess;
    aov_fix32_kernel<<<n_curves, kPrepThreads, 0, stream>>>(m, aux32, curves, n_curves);
    return cudaGetLastError();
}

cudaError_t launch_pack(const float* src_t, const float* src_m, const int64_t* src_off,
                        const CurveDesc* curves, uint32_t n_curves, float* dst_t, float* dst_m,
                        cudaStream_t stream) {
    if (n_curves == 0) return cudaSuccess;
    pack_kernel<<<n_curves, kPrepThreads, 0, stream>>>(src_t, src_m, src_off, curves, n_curves,
                                                       dst_t, dst_m);
    return cudaGetLastError();
}

cudaError_t launch_aov_mean(const float* m, CurveDesc* curves, uint32_t n_curves,
                            cudaStream_t stream) {
    if (n_curves == 0) return cudaSuccess;
    aov_mean_kernel<<<n_curves, kPrepThreads, 0, stream>>>(m, curves, n_curves);
    return cudaGetLastError();
}

cudaError_t launch_aov_fix_prep(const float* m, uint64_t* aux64, CurveDesc* curves,
                                uint32_t n_curves, uint32_t overlap, cudaStream_t stream) {
    if (n_curves == 0) return cudaSuccess;
    aov_fix_kernel<<<n_curves, kPrepThreads, 0, stream>>>(m, aux64, curves, n_curves, overlap);
    return cudaGetLastError();
}

}  // namespace pfk
