// pipe_peaks.cu -- measured per-SM throughput of the execution pipes the
// periodogram kernels are bound by (FP64 FMA and divide, FP32 FMA, MUFU
// sin/cos, f64<->f32 conversion, shared-memory atomics).  These are the
// roofline denominators for kernels that are neither HBM- nor tensor-bound.
//
// Each probe runs a fixed number of independent operation chains per thread
// on a full grid (4 CTAs of 256 threads per SM) and records, per CTA, the SM
// cycle count from clock64(), so the result is ops per SM per cycle,
// independent of the clock the GPU happened to run at.  Wall time (CUDA
// events) is also returned so ops/s at the observed clock can be reported.
//
// C entry point: pfpk_measure(int device, pfpk_result* out, int n).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

namespace {

constexpr int kThreads = 256;
constexpr int kIters = 65536;

struct Probe {
    long long* cycles;  // per CTA: SM cycles
    long long* nanos;   // per CTA: global-timer nanoseconds
    float* sink;
};

__device__ __forceinline__ long long gtimer() {
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void record(const Probe& p, long long t0, long long g0, float v) {
    __syncthreads();
    if (threadIdx.x == 0) {
        p.cycles[blockIdx.x] = clock64() - t0;
        p.nanos[blockIdx.x] = gtimer() - g0;
    }
    if (v == 1234.5f) p.sink[blockIdx.x] = v;  // keep results live
}

// 8 independent FFMA chains per thread.
__global__ void k_ffma(Probe p, float a, float b) {
    float x[8];
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = threadIdx.x * 1e-3f + j;
    __syncthreads();
    long long t0 = clock64();
    long long g0 = gtimer();
#pragma unroll 4
    for (int i = 0; i < kIters; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) x[j] = __fmaf_rn(x[j], a, b);
    }
    float s = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) s += x[j];
    record(p, t0, g0, s);
}

// 8 independent DFMA chains per thread.
__global__ void k_dfma(Probe p, double a, double b) {
    double x[8];
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = threadIdx.x * 1e-3 + j;
    __syncthreads();
    long long t0 = clock64();
    long long g0 = gtimer();
#pragma unroll 2
    for (int i = 0; i < kIters / 4; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) x[j] = __fma_rn(x[j], a, b);
    }
    double s = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) s += x[j];
    record(p, t0, g0, (float)s);
}

// IEEE double division with a varying numerator (4 chains).
__global__ void k_ddiv(Probe p, double d) {
    double x[4];
#pragma unroll
    for (int j = 0; j < 4; j++) x[j] = 1.0 + threadIdx.x * 1e-3 + j;
    __syncthreads();
    long long t0 = clock64();
    long long g0 = gtimer();
    for (int i = 0; i < kIters / 64; i++) {
#pragma unroll
        for (int j = 0; j < 4; j++) x[j] = x[j] / d + 1.0;
    }
    double s = 0;
#pragma unroll
    for (int j = 0; j < 4; j++) s += x[j];
    record(p, t0, g0, (float)s);
}

// floor of a double (4 chains), plus the add that keeps the chain going.
__global__ void k_dfloor(Probe p, double a) {
    double x[8];
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = 1.5 + threadIdx.x * 1e-3 + j;
    __syncthreads();
    long long t0 = clock64();
    long long g0 = gtimer();
    for (int i = 0; i < kIters / 8; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) x[j] = floor(x[j]) + a;
    }
    double s = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) s += x[j];
    record(p, t0, g0, (float)s);
}

// f64 -> f32 -> f64 round trips (8 chains): two conversions per step.
__global__ void k_cvt(Probe p, float a) {
    double x[8];
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = 1.5 + threadIdx.x * 1e-3 + j;
    __syncthreads();
    long long t0 = clock64();
    long long g0 = gtimer();
    for (int i = 0; i < kIters / 8; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) x[j] = (double)(__double2float_rn(x[j]) * a);
    }
    double s = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) s += x[j];
    record(p, t0, g0, (float)s);
}

// MUFU sin + cos (8 chains).
__global__ void k_mufu(Probe p, float a) {
    float x[8];
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = threadIdx.x * 1e-3f + j;
    __syncthreads();
    long long t0 = clock64();
    long long g0 = gtimer();
    for (int i = 0; i < kIters / 8; i++) {
#pragma unroll
        for (int j = 0; j < 8; j++) x[j] = __sinf(x[j]) + __cosf(x[j] * a);
    }
    float s = 0;
#pragma unroll
    for (int j = 0; j < 8; j++) s += x[j];
    record(p, t0, g0, s);
}

// Shared atomic add into this thread's own column (no contention, no bank
// conflicts): the privatised-histogram update.  nbins is a power of two.
template <typename T>
__global__ void k_atoms_private(Probe p, int nbins, T inc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* h = reinterpret_cast<T*>(smem_raw);
    for (int i = threadIdx.x; i < nbins * kThreads; i += kThreads) h[i] = T(0);
    __syncthreads();
    const unsigned mask = nbins - 1;
    const unsigned lane4 = threadIdx.x >> 2;
    long long t0 = clock64();
    long long g0 = gtimer();
    for (int i = 0; i < kIters / 4; i++) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            unsigned b = (i * 5u + j * 11u + lane4) & mask;
            atomicAdd(&h[b * kThreads + threadIdx.x], inc);
        }
    }
    __syncthreads();
    record(p, t0, g0, (float)h[threadIdx.x]);
}

// Shared u32 atomic increment into one histogram per warp (lanes contend and
// conflict on banks as a real histogram does).  nbins is a power of two.
__global__ void k_atoms_warp(Probe p, int nbins) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned* h = reinterpret_cast<unsigned*>(smem_raw) + (threadIdx.x / 32) * nbins;
    for (int i = threadIdx.x; i < nbins * (kThreads / 32); i += kThreads)
        reinterpret_cast<unsigned*>(smem_raw)[i] = 0;
    __syncthreads();
    const unsigned mask = nbins - 1;
    const unsigned salt = (threadIdx.x * 2654435761u) >> 20;
    long long t0 = clock64();
    long long g0 = gtimer();
    for (int i = 0; i < kIters / 4; i++) {
#pragma unroll
        for (int j = 0; j < 4; j++) {
            unsigned b = ((i * 37u + j * 101u) ^ salt) & mask;
            atomicAdd(&h[b], 1u);
        }
    }
    __syncthreads();
    record(p, t0, g0, (float)h[threadIdx.x & mask]);
}

}  // namespace

extern "C" {

typedef struct {
    char name[32];
    double ops_per_clk_per_sm;  // lane operations per SM cycle (clock64)
    double ops_per_s;           // lane operations per second, whole GPU
    double sm_mhz;              // SM clock seen by the probe (clock64 / globaltimer)
} pfpk_result;

// Returns the number of results written, or a negative value on error.
int pfpk_measure(int device, pfpk_result* out, int n_out) {
    if (cudaSetDevice(device) != cudaSuccess) return -1;
    int n_sm = 0;
    cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device);
    const int ctas = n_sm * 4;
    long long *d_cyc, *d_ns;
    float* d_sink;
    if (cudaMalloc(&d_cyc, ctas * sizeof(long long)) != cudaSuccess) return -2;
    if (cudaMalloc(&d_ns, ctas * sizeof(long long)) != cudaSuccess) return -2;
    if (cudaMalloc(&d_sink, ctas * sizeof(float)) != cudaSuccess) return -2;
    Probe p{d_cyc, d_ns, d_sink};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    long long* h_cyc = new long long[ctas];
    long long* h_ns = new long long[ctas];
    int k = 0;

    auto run = [&](const char* name, double ops_per_thread, auto launch) {
        if (k >= n_out) return;
        launch();  // warm-up
        cudaEventRecord(e0);
        launch();
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaMemcpy(h_cyc, d_cyc, ctas * sizeof(long long), cudaMemcpyDeviceToHost);
        cudaMemcpy(h_ns, d_ns, ctas * sizeof(long long), cudaMemcpyDeviceToHost);
        double cyc = 0, ns = 0;
        for (int i = 0; i < ctas; i++) {
            cyc += (double)h_cyc[i];
            ns += (double)h_ns[i];
        }
        const double mhz = cyc / ns * 1e3;
        const double total = ops_per_thread * kThreads * (double)ctas;
        pfpk_result& r = out[k++];
        snprintf(r.name, sizeof(r.name), "%s", name);
        r.ops_per_s = total / (ms * 1e-3);
        r.sm_mhz = mhz;
        r.ops_per_clk_per_sm = r.ops_per_s / (mhz * 1e6) / n_sm;
    };

    run("ffma", 8.0 * kIters, [&] { k_ffma<<<ctas, kThreads>>>(p, 0.999f, 1e-3f); });
    run("dfma", 8.0 * (kIters / 4), [&] { k_dfma<<<ctas, kThreads>>>(p, 0.999, 1e-3); });
    run("ddiv", 4.0 * (kIters / 64), [&] { k_ddiv<<<ctas, kThreads>>>(p, 1.0001); });
    run("dfloor+dadd", 8.0 * (kIters / 8), [&] { k_dfloor<<<ctas, kThreads>>>(p, 0.25); });
    run("cvt_f64_f32_pair", 8.0 * (kIters / 8), [&] { k_cvt<<<ctas, kThreads>>>(p, 1.0f); });
    run("mufu_sin+cos", 16.0 * (kIters / 8), [&] { k_mufu<<<ctas, kThreads>>>(p, 0.5f); });
    // Shared-memory sizes keep 4 CTAs resident per SM (<= 56 KB each).
    cudaFuncSetAttribute(k_atoms_private<unsigned>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, 32 * kThreads * 4);
    cudaFuncSetAttribute(k_atoms_private<float>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, 32 * kThreads * 4);
    cudaFuncSetAttribute(k_atoms_private<unsigned long long>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, 16 * kThreads * 8);
    run("atoms_u32_private", 4.0 * (kIters / 4), [&] {
        k_atoms_private<unsigned><<<ctas, kThreads, 32 * kThreads * 4>>>(p, 32, 1u);
    });
    run("atoms_u64_private", 4.0 * (kIters / 4), [&] {
        k_atoms_private<unsigned long long><<<ctas, kThreads, 16 * kThreads * 8>>>(p, 16, 1ull);
    });
    run("atoms_f32_private", 4.0 * (kIters / 4), [&] {
        k_atoms_private<float><<<ctas, kThreads, 32 * kThreads * 4>>>(p, 32, 1.0f);
    });
    run("atoms_u32_warp128", 4.0 * (kIters / 4), [&] {
        k_atoms_warp<<<ctas, kThreads, 128 * 8 * 4>>>(p, 128);
    });

    cudaError_t err = cudaDeviceSynchronize();
    delete[] h_cyc;
    delete[] h_ns;
    cudaFree(d_cyc);
    cudaFree(d_ns);
    cudaFree(d_sink);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return err == cudaSuccess ? k : -3;
}

}  // extern "C"
