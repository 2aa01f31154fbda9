// pf_noalloc.cu -- Lomb-Scargle periodograms + top-N peak search on device
// pointers, allocating nothing.
//
// Who needs this: callers that may not call cudaMalloc at the point where
// they want periodogram peaks -- code running inside a framework that owns
// every byte of device memory through its own pool (a cudaMalloc there can
// fail or fragment the pool), code on a latency-critical path where
// cudaMalloc's implicit device synchronisation is unacceptable, and callers
// with a fixed memory budget decided up front.  The regular entry points
// grow per-context buffers with cudaMalloc on demand; this one uses a single
// file-scope device array instead, whose size is fixed when the library is
// loaded.
//
// Scratch: kScratchBytes (32 MiB) of device memory in g_scratch, held by
// every GPU that loads this library until the process exits.  It holds the
// batch description, a packed copy of the curves, the batch's max |t| and
// the periodograms; a call whose layout does not fit is rejected with
// PF_EINVAL and a message giving both sizes.  Host-side batch metadata is
// staged through a static 1 MiB host buffer (at most ~18 000 curves).
//
// Rules for callers:
//  - The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture.  The address is kept per device and CUDA
//    context: after cudaDeviceReset, or under another context, the next call
//    looks it up again (and should likewise come before any capture).
//  - Every call shares the one array and leaves its contents behind: calls
//    whose GPU work overlaps (different streams, or host threads with
//    different streams) race on it.  Order them on one stream.
//  - The call enqueues work on `stream` and returns; outputs are ready when
//    the stream reaches that point.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/pf.h"
#include "pf_launch.h"
#include "pf_types.h"

using namespace pfk;

namespace {

constexpr size_t kScratchBytes = 32ull << 20;
constexpr size_t kMetaBytes = 1ull << 20;
constexpr int kMaxDevices = 64;
constexpr int kBlock = 256;  // LS launch shape (no histogram)

__device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;                       // guards g_meta, g_ptr and g_ctx
unsigned char* g_ptr[kMaxDevices];     // g_scratch's device address per device
CUcontext g_ctx[kMaxDevices];          // the context that address belongs to

// The calling thread's current CUDA context (the driver's cuCtxGetCurrent,
// reached through the runtime; NULL if it cannot be had).
CUcontext current_context() {
    using Fn = CUresult (*)(CUcontext*);
    static Fn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<Fn>(f);
    }();
    CUcontext c = nullptr;
    if (fn && fn(&c) != CUDA_SUCCESS) c = nullptr;
    return c;
}
alignas(256) unsigned char g_meta[kMetaBytes];

// Write the message into the caller's buffer (if any) and return `code`.
int fail(char* err, uint64_t err_len, int code, const char* fmt, ...)
    __attribute__((format(printf, 4, 5)));
int fail(char* err, uint64_t err_len, int code, const char* fmt, ...) {
    if (err && err_len > 0) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(err, (size_t)err_len, fmt, ap);
        va_end(ap);
    }
    return code;
}

inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Work items in launch order: curve-major, then period derivative, then
// tiles of kBlock periods (the same decomposition the fold kernel expects),
// and the curve order of the persistent folds' queue (input order).
__global__ void work_gen_kernel(WorkItem* __restrict__ work, uint32_t* __restrict__ order,
                                uint32_t n_curves, uint32_t n_work, uint32_t n_pdt,
                                uint32_t n_per) {
    const uint32_t tiles = (n_per + kBlock - 1) / kBlock;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n_work;
         k += gridDim.x * blockDim.x) {
        if (k < n_curves) order[k] = k;
        const uint32_t per_curve = n_pdt * tiles;
        const uint32_t c = k / per_curve;
        const uint32_t r = k % per_curve;
        const uint32_t d = r / tiles;
        const uint32_t t = r % tiles;
        WorkItem w;
        w.curve = c;
        w.pdt = d;
        w.p0 = t * kBlock;
        w.np = min((uint32_t)kBlock, n_per - t * kBlock);
        work[k] = w;
    }
}

}  // namespace

extern "C" int pf_ls_peaks_dev_noalloc(const float* d_times, const float* d_mags,
                                       const int64_t* offsets, uint64_t n_curves,
                                       const float* d_periods, uint64_t n_per,
                                       const float* d_pdts, uint64_t n_pdt, uint32_t n_peaks,
                                       uint32_t min_distance, int mode, int64_t* d_out_idx,
                                       float* d_out_val, void* stream, char* err,
                                       uint64_t err_len) {
    if (err && err_len > 0) err[0] = '\0';
    if (n_curves == 0 || n_peaks == 0) return PF_OK;
    if (!offsets || !d_periods || !d_pdts || !d_out_idx || !d_out_val)
        return fail(err, err_len, PF_EINVAL, "NULL argument");
    if (n_per == 0 || n_pdt == 0) return fail(err, err_len, PF_EINVAL, "empty trial grid");
    if (n_per > 0xFFFFFFFFull || n_pdt > 0xFFFFull || n_curves > 0x7FFFFFFFull)
        return fail(err, err_len, PF_EINVAL, "grid or batch too large");
    if (offsets[n_curves] > 0 && (!d_times || !d_mags))
        return fail(err, err_len, PF_EINVAL, "d_times/d_mags is NULL");

    // Layout of the scratch array (256-byte aligned sections).
    const size_t meta_curves = n_curves * sizeof(CurveDesc);
    const size_t meta_srcoff = n_curves * sizeof(int64_t);
    const size_t meta_bytes = align256(meta_curves) + align256(meta_srcoff);
    size_t total_pts = 0;
    for (uint64_t c = 0; c < n_curves; c++) {
        if (offsets[c + 1] < offsets[c] || offsets[c] < 0)
            return fail(err, err_len, PF_EINVAL, "offsets must be non-decreasing and non-negative");
        const uint64_t len = (uint64_t)(offsets[c + 1] - offsets[c]);
        if (len > 0xFFFFFFFFull) return fail(err, err_len, PF_EINVAL, "curve %llu too long", (unsigned long long)c);
        total_pts += (len + 3) & ~(uint64_t)3;
    }
    const uint64_t tiles = (n_per + kBlock - 1) / kBlock;
    const uint64_t n_work = n_curves * n_pdt * tiles;
    if (n_work > 0x7FFFFFFFull) return fail(err, err_len, PF_EINVAL, "too much work for one launch");
    const size_t o_tmax = 0;
    const size_t o_queue = 128;  // queue counter of the persistent folds
    const size_t o_meta = 256;
    const size_t o_work = o_meta + meta_bytes;
    const size_t o_order = align256(o_work + n_work * sizeof(WorkItem));
    const size_t o_t = align256(o_order + n_curves * sizeof(uint32_t));
    const size_t o_m = align256(o_t + total_pts * 4);
    const size_t o_pg = align256(o_m + total_pts * 4);
    const size_t need = o_pg + (size_t)n_curves * n_per * n_pdt * 4;
    if (need > kScratchBytes)
        return fail(err, err_len, PF_EINVAL,
                    "batch needs %zu bytes of scratch; this entry point has %zu (use pf_ls_peaks "
                    "or pf_ls_dev, which allocate)",
                    need, kScratchBytes);
    if (meta_bytes > kMetaBytes)
        return fail(err, err_len, PF_EINVAL, "batch metadata needs %zu bytes; the limit is %zu", meta_bytes,
                    kMetaBytes);

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(err, err_len, PF_ECUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(err, err_len, PF_EUNSUPPORTED, "device index %d", dev);

    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ptr[dev] || g_ctx[dev] != current_context()) {
        // Set-up on this device (with it current), once per context: the
        // host-side name g_scratch is only a stand-in; the kernels need its
        // address, which a new context (after cudaDeviceReset) moves.
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess)
            return fail(err, err_len, PF_ECUDA, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        g_ptr[dev] = static_cast<unsigned char*>(p);
        g_ctx[dev] = current_context();
    }
    unsigned char* base = g_ptr[dev];
    cudaStream_t s = (cudaStream_t)stream;

    // Curve descriptors (padded layout) and source offsets, staged on the
    // host in the static buffer; a pageable copy consumes it before returning.
    CurveDesc* hc = reinterpret_cast<CurveDesc*>(g_meta);
    int64_t* hs = reinterpret_cast<int64_t*>(g_meta + align256(meta_curves));
    size_t run = 0;
    for (uint64_t c = 0; c < n_curves; c++) {
        CurveDesc d;
        memset(&d, 0, sizeof(d));
        d.off = (int64_t)run;
        d.n = (uint32_t)(offsets[c + 1] - offsets[c]);
        hc[c] = d;
        hs[c] = offsets[c];
        run += (d.n + 3u) & ~3u;
    }
    if ((e = cudaMemcpyAsync(base + o_meta, g_meta, meta_bytes, cudaMemcpyHostToDevice, s)) !=
        cudaSuccess)
        return fail(err, err_len, PF_ECUDA, "metadata copy: %s", cudaGetErrorString(e));

    CurveDesc* dcurves = reinterpret_cast<CurveDesc*>(base + o_meta);
    const int64_t* dsrc = reinterpret_cast<const int64_t*>(base + o_meta + align256(meta_curves));
    WorkItem* dwork = reinterpret_cast<WorkItem*>(base + o_work);
    float* pt = reinterpret_cast<float*>(base + o_t);
    float* pm = reinterpret_cast<float*>(base + o_m);
    float* pg = reinterpret_cast<float*>(base + o_pg);
    unsigned* tmax = reinterpret_cast<unsigned*>(base + o_tmax);

    uint32_t* dorder = reinterpret_cast<uint32_t*>(base + o_order);
    const int gen_blocks = (int)std::min<uint64_t>((n_work + 255) / 256, 4096);
    work_gen_kernel<<<gen_blocks, 256, 0, s>>>(dwork, dorder, (uint32_t)n_curves,
                                                (uint32_t)n_work, (uint32_t)n_pdt,
                                                (uint32_t)n_per);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return fail(err, err_len, PF_ECUDA, "work-list kernel: %s", cudaGetErrorString(e));
    if ((e = launch_pack(d_times, d_mags, dsrc, dcurves, (uint32_t)n_curves, pt, pm, s)) !=
        cudaSuccess)
        return fail(err, err_len, PF_ECUDA, "pack kernel: %s", cudaGetErrorString(e));
    // launch_tmax clears the max-|t| word before reducing into it.
    if ((e = launch_tmax(pt, total_pts, tmax, s)) != cudaSuccess)
        return fail(err, err_len, PF_ECUDA, "max|t| kernel: %s", cudaGetErrorString(e));

    int n_sm = 0;
    if ((e = cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return fail(err, err_len, PF_ECUDA, "device attribute: %s", cudaGetErrorString(e));
    FoldConfig cfg{};
    cfg.n_sm = n_sm;
    cfg.kind = KIND_FOLD;
    cfg.algo = ALGO_LS;
    cfg.acc = 0;
    cfg.block = kBlock;
    cfg.ovl = false;
    const bool chosen = (mode & PF_MODE_CHOSEN) != 0;
    cfg.fold = chosen ? ((mode & PF_FOLD_EXACT) ? FOLD_EXACT : FOLD_DF) : FOLD_REF;
    if (mode & PF_FOLD_DF) cfg.fold = FOLD_DF;
    if (mode & PF_FOLD_F32) cfg.fold = FOLD_F32;

    FoldParams p;
    memset(&p, 0, sizeof(p));
    p.t = pt;
    p.m = pm;
    p.curves = dcurves;
    p.work = dwork;
    p.periods = d_periods;
    p.pdts = d_pdts;
    p.out = pg;
    p.n_per = (uint32_t)n_per;
    p.n_pdt = (uint32_t)n_pdt;
    p.n_phase = 1;
    p.n_mag = 1;
    p.p_overlap = 1;
    p.m_overlap = 1;
    p.tmax_bits = tmax;
    p.q.order = dorder;
    p.q.n_work = (uint32_t)n_work;
    p.q.next = reinterpret_cast<unsigned*>(base + o_queue);
    e = (mode & PF_SEM_CPU) ? launch_fold_cpusem(cfg, p, (uint32_t)n_work, s)
                            : launch_fold_cudasem(cfg, p, (uint32_t)n_work, s);
    if (e != cudaSuccess) return fail(err, err_len, PF_ECUDA, "LS kernel: %s", cudaGetErrorString(e));
    if ((e = launch_peaks(pg, n_curves, n_per * n_pdt, n_peaks, min_distance, 1, d_out_idx,
                          d_out_val, s)) != cudaSuccess)
        return fail(err, err_len, PF_ECUDA, "peak kernel: %s", cudaGetErrorString(e));
    return PF_OK;
}
