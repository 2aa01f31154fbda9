// pf_api.cu -- the C ABI (include/pf.h): argument checks, packing, launch
// decomposition and the device pipeline
//     pack (host, pinned) -> one H2D copy -> preparation kernels ->
//     fused fold/bin/statistic kernel (one launch for the plain form, one
//     per curve-length class with its tuned shape for the chosen form) ->
//     periodogram D2H, or peak search / row statistics on the device and a
//     D2H of those only.  Peak calls with PF_ASYNC return once their work
//     is queued; pf_wait collects them.
//
// Compared with the reference's drivers (periodfind/cuda/ce.cu:420-562,
// aov.cu:429-576, ls.cu:232-359), which allocate and free every buffer per
// call, copy each curve with its own pageable memcpy, launch one or two
// kernels per curve and exit() on any CUDA error, this driver keeps
// grow-only device and pinned buffers in the context, moves the whole batch
// in one copy, launches a handful of kernels for the whole batch and
// reports errors as status codes.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <limits>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/pf.h"
#include "pf_launch.h"
#include "pf_types.h"

using namespace pfk;

namespace {

struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
};

struct PinnedBuf {
    void* p = nullptr;
    size_t cap = 0;
};

thread_local std::string g_create_error;

// An NVTX range around one stage of a call (pack, copies, preparation,
// fold / bin kernels, statistics, peak search), seen by a profiler's
// timeline; without a profiler attached it costs a function-pointer check.
struct Stage {
    explicit Stage(const char* name) { nvtxRangePushA(name); }
    ~Stage() { nvtxRangePop(); }
    Stage(const Stage&) = delete;
    Stage& operator=(const Stage&) = delete;
};

// Host threads kept by a context for the packing of host-pointer calls:
// run() hands the tasks of one job to the workers and the calling thread,
// which take them in turn; idle workers wait on a condition variable.
// Threads are created on first use (a thread start costs tens of
// microseconds, more than packing a small batch).  A task ticket carries
// the job number, so a worker that wakes after its job has finished takes
// nothing from the next one, and the caller waits for its tasks, not for
// every worker to wake.  One job at a time (a context is used by one host
// thread at a time).
class WorkerPool {
  public:
    WorkerPool() = default;
    WorkerPool(const WorkerPool&) = delete;
    WorkerPool& operator=(const WorkerPool&) = delete;
    ~WorkerPool() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (std::thread& t : threads_) t.join();
    }

    // fn(k) for every k < n_tasks, on at most `width` threads (the caller
    // included); returns when all tasks have finished.
    void run(unsigned n_tasks, unsigned width, const std::function<void(unsigned)>& fn) {
        width = std::min(width, n_tasks);
        if (width <= 1) {
            for (unsigned k = 0; k < n_tasks; k++) fn(k);
            return;
        }
        while (threads_.size() + 1 < width) {
            const uint32_t g = gen_;  // the new worker waits for the next job
            try {
                threads_.emplace_back([this, g] { work(g); });
            } catch (...) {
                break;  // no more threads to be had: run with those there are
            }
        }
        if (threads_.empty()) {
            for (unsigned k = 0; k < n_tasks; k++) fn(k);
            return;
        }
        uint32_t g;
        {
            std::lock_guard<std::mutex> lk(mu_);
            g = ++gen_;
            fn_ = &fn;
            n_tasks_ = n_tasks;
            done_.store(0, std::memory_order_relaxed);
            ticket_.store((uint64_t)g << 32, std::memory_order_release);
        }
        cv_.notify_all();
        take(g, &fn, n_tasks);
        while (done_.load(std::memory_order_acquire) < n_tasks) std::this_thread::yield();
    }

  private:
    // Tasks of job g until none is left (or a newer job has started).
    void take(uint32_t g, const std::function<void(unsigned)>* fn, unsigned n) {
        for (;;) {
            uint64_t v = ticket_.load(std::memory_order_acquire);
            do {
                if ((uint32_t)(v >> 32) != g || (uint32_t)v >= n) return;
            } while (!ticket_.compare_exchange_weak(v, v + 1, std::memory_order_acq_rel));
            (*fn)((unsigned)(uint32_t)v);
            done_.fetch_add(1, std::memory_order_release);
        }
    }
    void work(uint32_t seen) {
        for (;;) {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
            if (stop_) return;
            seen = gen_;
            const std::function<void(unsigned)>* fn = fn_;
            const unsigned n = n_tasks_;
            lk.unlock();
            take(seen, fn, n);
        }
    }

    std::vector<std::thread> threads_;
    std::mutex mu_;
    std::condition_variable cv_;
    const std::function<void(unsigned)>* fn_ = nullptr;
    unsigned n_tasks_ = 0;
    uint32_t gen_ = 0;                 // job number (guarded by mu_)
    std::atomic<uint64_t> ticket_{0};  // (job number << 32) | next task
    std::atomic<unsigned> done_{0};    // tasks of the current job finished
    bool stop_ = false;
};

}  // namespace

struct pf_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;   // around the fold kernel
    cudaEvent_t ev_staged = nullptr;            // staging block copied out
    cudaEvent_t ev_done = nullptr;              // the last call's work done
    bool staged_pending = false, done_recorded = false, timed_pending = false;
    std::string err;
    DevBuf d_in, d_aux32, d_aux64, d_out, d_pidx, d_pval, d_pack, d_misc, d_stamps, d_stat;
    DevBuf d_bins;  // pf_bin_counts: raw bin counts per cell
    // pf_prepare_mags_dev: the curve offsets on the device, and the event
    // after the last kernel that read them (the buffer is rewritten only
    // once that kernel is done).
    DevBuf d_prep;
    cudaEvent_t ev_prep = nullptr;
    bool prep_pending = false;
    // PF_TIMING: the curve of each work item of the last timed launch, and
    // the stream it ran on.
    std::vector<uint32_t> stamp_curves;   // curve of each stamped work item
    uint64_t stamp_n_curves = 0;
    cudaStream_t stamp_stream = nullptr;
    PinnedBuf h_in;
    // Host-pointer calls alternate between two device input blocks (d_in,
    // d_in2) and copy on copy_stream, so that a call's inputs cross PCIe
    // while the previous call's kernels run.  ev_in_free[i] follows the last
    // kernel that read block i, ev_copied[i] the copy into it.  cur_slot is
    // the block of the call being finished (-1: not a host call, which
    // frees both).
    DevBuf d_in2;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t ev_in_free[2] = {nullptr, nullptr};
    cudaEvent_t ev_copied[2] = {nullptr, nullptr};
    int in_slot = 0, cur_slot = -1;
    // Small results (statistics, best cells, synchronous peaks) land here
    // and are copied into the caller's arrays after the synchronisation: a
    // device-to-host copy into pageable memory costs more than the memcpy.
    PinnedBuf h_res;
    struct HostCopy {
        void* dst;
        const void* src;
        size_t n;
    };
    std::vector<HostCopy> res_copies;  // h_res -> caller, after the synchronisation
    WorkerPool pool;
    uint64_t launches = 0;
    double last_ms = -1.0;
    int n_sm = 0;
    size_t smem_optin = 0;
    // Autotuner: launch shape per (computation, length class), measured on
    // the device the first time the key is met (see tuned_config).
    struct Tuned {
        int kind;  // KIND_* of the winner (LS on a frequency grid: the trig form)
        int block;
        bool persist;
        int rounds;
        float ms;        // sample time of the winner
        float ms_worst;  // and of the slowest candidate
        uint32_t candidates;
    };
    std::map<std::string, Tuned> tuned;
    // PF_ASYNC peak calls not yet collected by pf_wait, oldest first.  Each
    // copies its peaks into its own pinned block; the event follows the copy.
    struct Pending {
        PinnedBuf res;
        cudaEvent_t done = nullptr;
        int64_t* out_idx = nullptr;
        float* out_val = nullptr;
        size_t n = 0;       // peak entries to hand over
        bool work = false;  // the call queued device work
    };
    static constexpr int kMaxPending = 2;
    Pending pend[kMaxPending];
    int pend_head = 0, pend_count = 0;
};

namespace {

int fail(pf_ctx* ctx, int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (ctx) ctx->err = buf;
    return code;
}

int cuda_fail(pf_ctx* ctx, cudaError_t e, const char* what) {
    return fail(ctx, PF_ECUDA, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

#define PF_CUDA(call, what)                                   \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, what); \
    } while (0)

// Calls on a context share its device buffers, and may run on different
// streams (host-pointer calls on the context's stream, device-pointer calls
// on the caller's).  Each call orders its first use of the buffers after
// the previous call's last (order_after_previous) and marks its own end
// (mark_done), so a call never overwrites inputs, descriptors or queue
// counters that an earlier call's kernels still read.  The one exception is
// a host call's input copy, which goes to the input block the previous call
// did not use and waits only for that block's last reader (ev_in_free).
int order_after_previous(pf_ctx* ctx, cudaStream_t s) {
    if (ctx->done_recorded) PF_CUDA(cudaStreamWaitEvent(s, ctx->ev_done, 0), "stream wait");
    return PF_OK;
}

int mark_done(pf_ctx* ctx, cudaStream_t s) {
    PF_CUDA(cudaEventRecord(ctx->ev_done, s), "event");
    ctx->done_recorded = true;
    // The input blocks this call's kernels read are free once they are
    // done: a host call's own block; both for any other call.
    for (int i = 0; i < 2; i++)
        if (ctx->cur_slot < 0 || ctx->cur_slot == i)
            PF_CUDA(cudaEventRecord(ctx->ev_in_free[i], s), "event");
    ctx->cur_slot = -1;
    return PF_OK;
}

// Marks a host call's end on its stream when it returns early, after its
// copy or kernels were queued: the input blocks count as in use until then.
struct CallEnd {
    pf_ctx* ctx;
    cudaStream_t s;
    bool armed = true;
    ~CallEnd() {
        if (!armed) return;
        cudaEventRecord(ctx->ev_done, s);
        ctx->done_recorded = true;
        cudaEventRecord(ctx->ev_in_free[0], s);
        cudaEventRecord(ctx->ev_in_free[1], s);
        ctx->cur_slot = -1;
        cudaGetLastError();
    }
};

int ensure_dev(pf_ctx* ctx, DevBuf& b, size_t bytes) {
    if (bytes <= b.cap) return PF_OK;
    // The old block may still be read by the previous call's kernels.
    if (b.p && ctx->done_recorded) cudaEventSynchronize(ctx->ev_done);
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t want = std::max(bytes, (size_t)256);
    want = (want + (want >> 3) + 255) & ~(size_t)255;  // 12.5% headroom
    cudaError_t e = cudaMalloc(&b.p, want);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, PF_ENOMEM, "device allocation of %zu bytes failed: %s", want,
                    cudaGetErrorString(e));
    }
    b.cap = want;
    return PF_OK;
}

int ensure_pinned(pf_ctx* ctx, PinnedBuf& b, size_t bytes) {
    if (bytes <= b.cap) return PF_OK;
    if (b.p) cudaFreeHost(b.p);
    b.p = nullptr;
    b.cap = 0;
    size_t want = std::max(bytes, (size_t)4096);
    want = (want + (want >> 3) + 4095) & ~(size_t)4095;
    cudaError_t e = cudaHostAlloc(&b.p, want, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, PF_ENOMEM, "pinned allocation of %zu bytes failed: %s", want,
                    cudaGetErrorString(e));
    }
    b.cap = want;
    return PF_OK;
}

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// numpy's pairwise float32 summation (the add.reduce behind np.mean of a
// contiguous float32 array; numpy/_core/src/umath/loops_utils.h.src,
// pairwise_sum): fewer than 8 elements are added in order starting from
// -0.0; up to 128 elements go to eight interleaved accumulators, combined as
// ((r0 + r1) + (r2 + r3)) + ((r4 + r5) + (r6 + r7)), then the remainder in
// order; a longer range splits at n / 2 rounded down to a multiple of 8 and
// the two halves' sums are added.  This unit is built without contraction,
// so every addition is one IEEE float32 rounding, as in numpy.
float numpy_pairwise_sum(const float* a, uint64_t n) {
    if (n < 8) {
        float res = -0.0f;
        for (uint64_t i = 0; i < n; i++) res += a[i];
        return res;
    }
    if (n <= 128) {
        float r[8];
        for (int k = 0; k < 8; k++) r[k] = a[k];
        uint64_t i = 8;
        for (; i < n - (n % 8); i += 8)
            for (int k = 0; k < 8; k++) r[k] += a[i + k];
        float res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; i++) res += a[i];
        return res;
    }
    uint64_t n2 = n / 2;
    n2 -= n2 % 8;
    return numpy_pairwise_sum(a, n2) + numpy_pairwise_sum(a + n2, n - n2);
}

// Run fn(c) for every curve, on several host threads when the batch holds
// more than 2^20 points (curves interleaved across the threads).
template <class F>
void for_each_curve(uint64_t n_curves, uint64_t total_points, F& fn) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const unsigned nthr = total_points > (1u << 20) ? hw : 1u;
    if (nthr == 1) {
        for (uint64_t c = 0; c < n_curves; c++) fn(c);
        return;
    }
    std::vector<std::thread> th;
    for (unsigned w = 0; w < nthr; w++)
        th.emplace_back([&, w] {
            for (uint64_t c = w; c < n_curves; c += nthr) fn(c);
        });
    for (auto& t : th) t.join();
}

// The packing of a host-pointer call split into tasks for the context's
// worker threads: consecutive curve ranges of about equal point counts
// (first[k] .. first[k+1]), on one thread per 16k points up to 16.
struct CurveTasks {
    unsigned width = 1;
    std::vector<uint64_t> first;
    unsigned count() const { return (unsigned)first.size() - 1; }
};

CurveTasks curve_tasks(const std::vector<int64_t>& off, uint64_t total_pts) {
    constexpr uint64_t kPointsPerThread = 16384;
    CurveTasks T;
    const uint64_t n_curves = off.size();
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    T.width = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(hw, total_pts / kPointsPerThread));
    const uint64_t n_tasks = std::max<uint64_t>(1, std::min<uint64_t>(n_curves, 4ull * T.width));
    T.first.resize(n_tasks + 1);
    for (uint64_t k = 0; k < n_tasks; k++)
        T.first[k] = (uint64_t)(std::lower_bound(off.begin(), off.end(),
                                                 (int64_t)(k * total_pts / n_tasks)) -
                                off.begin());
    T.first[0] = 0;
    T.first[n_tasks] = n_curves;
    return T;
}

// The reference's normalize=True preparation of one curve
// (periodfind/_utils.py:39-45) with numpy's float32 arithmetic:
// ((m - min) / (max - min)) * 0.999 + 5e-4, out may equal m.
void normalize_curve(const float* m, uint64_t n, float* o) {
    // Per curve: numpy's float32 min / max (NaN propagates), then
    // ((m - lo) / (hi - lo)) * 0.999f + 5e-4f in single precision, one
    // rounding per operation, as numpy evaluates the same expression.
    float lo = m[0], hi = m[0];
    bool nan = std::isnan(m[0]);
    uint64_t i = 1;
    if (n >= 16) {
        // Eight interleaved running minima / maxima, which the compiler
        // turns into SIMD min / max.  Without NaN the result is the exact
        // minimum and maximum whatever the order; only the sign of a
        // zero extreme may differ, and lo, hi enter the output solely
        // through m - lo and hi - lo, whose values it does not change.
        float l[8], h[8];
        int bad[8];
        for (int k = 0; k < 8; k++) {
            l[k] = h[k] = m[k];
            bad[k] = 0;
        }
        for (i = 0; i + 8 <= n; i += 8)
            for (int k = 0; k < 8; k++) {
                const float v = m[i + k];
                bad[k] |= (v != v);
                l[k] = v < l[k] ? v : l[k];
                h[k] = v > h[k] ? v : h[k];
            }
        for (int k = 0; k < 8; k++) {
            nan |= bad[k] != 0;
            lo = l[k] < lo ? l[k] : lo;
            hi = h[k] > hi ? h[k] : hi;
        }
    }
    for (; i < n; i++) {
        const float v = m[i];
        nan |= std::isnan(v);
        lo = v < lo ? v : lo;
        hi = v > hi ? v : hi;
    }
    if (nan) lo = hi = std::numeric_limits<float>::quiet_NaN();
    // This unit is built with -ffp-contract=off: no fused multiply-add.
    const float range = hi - lo;
    for (uint64_t i = 0; i < n; i++) o[i] = ((m[i] - lo) / range) * 0.999f + 5e-4f;
}

// The reference's center=True preparation of one curve
// (periodfind/_utils.py:35-37): np.mean of a float32 array is the pairwise
// float32 sum divided by the length in float32; then m - mean, one
// rounding per point.  out may equal m.
void center_curve(const float* m, uint64_t n, float* o) {
    const float mean = numpy_pairwise_sum(m, n) / (float)n;
    for (uint64_t i = 0; i < n; i++) o[i] = m[i] - mean;
}


// What one call computes.
struct Job {
    int algo = ALGO_CE;
    int mode = 0;
    uint64_t n_curves = 0;
    const float* periods = nullptr;  // host or device (see dev)
    uint64_t n_per = 0;
    const float* pdts = nullptr;
    uint64_t n_pdt = 0;
    uint32_t n_phase = 10, n_mag = 10, po = 1, mo = 1;
    // outputs
    float* out = nullptr;  // host periodogram, or device periodogram (dev)
    bool peaks = false;
    uint32_t n_peaks = 0, min_distance = 1;
    int64_t* out_idx = nullptr;
    float* out_val = nullptr;
    // 'stats' output on the device: per curve (mean, std, median, mad) into
    // out_stats and the n_top best cells into out_idx / out_val.
    bool stats = false;
    uint32_t n_top = 0;
    float* out_stats = nullptr;
    // pf_bin_counts: raw bin counts per cell ([curve][period][pdt][bins]).
    uint32_t* out_bins = nullptr;
    // pf_ls_fgrid: trial frequencies f0 + k * df (k < n_per), no periods
    // array, one period derivative (0).
    bool fgrid = false;
    double f0 = 0.0, df = 0.0;
};

// Bins per cell of a bin-count call: n_phase x n_mag (CE), n_phase (AOV).
size_t bins_per_cell(const Job& j) {
    return j.algo == ALGO_CE ? (size_t)j.n_phase * j.n_mag : (size_t)j.n_phase;
}

// Layout of the packed input block (host staging and its device copy).
struct Layout {
    std::vector<int64_t> off;  // per curve, in points (multiple of 4)
    std::vector<uint32_t> len;
    std::vector<uint32_t> order;  // queue kernels: curves longest first
    size_t total_pts = 0;      // padded
    size_t o_t = 0, o_m = 0, o_curves = 0, o_work = 0, o_periods = 0, o_pdts = 0, o_srcoff = 0;
    size_t o_tmax = 0;  // host-packed calls: max |t| of the batch (float bits)
    size_t bytes = 0;
    uint32_t n_work = 0;
    uint32_t max_len = 0;
};

bool use_cpu_semantics(int mode) { return (mode & PF_SEM_CPU) != 0; }

// The bin width the reference stores: CUDA keeps 1.0 / (float)n computed in
// double and rounded to float (ce.cu:34-35, aov.cu:24); Rust divides in f32
// (ce.rs:54-55, aov.rs:141).
float bin_size(uint32_t n, bool cpu_sem) {
    if (cpu_sem) return 1.0f / (float)n;
    return (float)(1.0 / static_cast<float>(n));
}

int validate_common(pf_ctx* ctx, const Job& j) {
    if (!ctx) return PF_EINVAL;
    if (j.fgrid) {
        if (j.algo != ALGO_LS || !(j.mode & PF_MODE_CHOSEN))
            return fail(ctx, PF_EUNSUPPORTED, "a frequency grid is for the chosen LS form only");
        if (j.mode & (PF_FOLD_F32 | PF_SEM_CPU))
            return fail(ctx, PF_EUNSUPPORTED,
                        "a frequency grid takes the split-precision or exact fold, CUDA arithmetic");
        const double last = j.f0 + (double)(j.n_per ? j.n_per - 1 : 0) * j.df;
        if (!std::isfinite(j.f0) || !std::isfinite(j.df) || !std::isfinite(last))
            return fail(ctx, PF_EINVAL, "frequency grid f0 = %g, df = %g is not finite", j.f0,
                        j.df);
    }
    if (j.n_curves > 0 && (j.n_per == 0 || j.n_pdt == 0)) return PF_OK;  // nothing to compute
    if (j.n_per > 0 && !j.periods && !j.fgrid) return fail(ctx, PF_EINVAL, "periods is NULL");
    if (j.n_pdt > 0 && !j.pdts && !j.fgrid) return fail(ctx, PF_EINVAL, "period_dts is NULL");
    if (j.n_per > 0xFFFFFFFFull || j.n_pdt > 0xFFFFull)
        return fail(ctx, PF_EINVAL, "grid too large (n_per %llu, n_pdt %llu)",
                    (unsigned long long)j.n_per, (unsigned long long)j.n_pdt);
    if (j.n_curves > 0x7FFFFFFFull) return fail(ctx, PF_EINVAL, "too many curves");
    if (j.algo == ALGO_CE || j.algo == ALGO_AOV) {
        if (j.n_phase < 1 || j.n_phase > 4096)
            return fail(ctx, PF_EINVAL, "n_phase must be in [1, 4096], got %u", j.n_phase);
        if (j.po < 1 || j.po > j.n_phase)
            return fail(ctx, PF_EINVAL, "phase overlap must be in [1, n_phase], got %u", j.po);
        if (j.algo == ALGO_AOV && j.n_phase < 2)
            return fail(ctx, PF_EINVAL, "AOV needs n_phase >= 2");
    }
    if (j.algo == ALGO_CE) {
        if (j.n_mag < 1 || j.n_mag > 4096)
            return fail(ctx, PF_EINVAL, "n_mag must be in [1, 4096], got %u", j.n_mag);
        if (j.mo < 1 || j.mo > j.n_mag)
            return fail(ctx, PF_EINVAL, "mag overlap must be in [1, n_mag], got %u", j.mo);
    }
    if (j.peaks && (!j.out_idx || !j.out_val) && j.n_peaks > 0)
        return fail(ctx, PF_EINVAL, "peak outputs are NULL");
    if (j.stats && (!j.out_stats || (j.n_top > 0 && (!j.out_idx || !j.out_val))))
        return fail(ctx, PF_EINVAL, "stats outputs are NULL");
    if (j.stats && j.n_per * j.n_pdt > 0 && stats_leaf_count((uint32_t)std::min<uint64_t>(
                                                   j.n_per * j.n_pdt, 0xFFFFFFFFull)) *
                                                   12ull > 200ull * 1024ull)
        return fail(ctx, PF_EUNSUPPORTED, "periodogram rows too long for the device statistics");
    if (!j.peaks && !j.stats && !j.out && j.n_curves > 0)
        return fail(ctx, PF_EINVAL, "out is NULL");
    return PF_OK;
}

int check_grid_host(pf_ctx* ctx, const Job& j) {
    for (uint64_t i = 0; i < (j.fgrid ? 0 : j.n_per); i++) {
        const float P = j.periods[i];
        if (!std::isfinite(P) || P == 0.0f)
            return fail(ctx, PF_EINVAL, "periods[%llu] = %g must be finite and non-zero",
                        (unsigned long long)i, (double)P);
    }
    for (uint64_t i = 0; i < j.n_pdt; i++) {
        if (!std::isfinite(j.pdts[i]))
            return fail(ctx, PF_EINVAL, "period_dts[%llu] is not finite", (unsigned long long)i);
    }
    return PF_OK;
}

// Warps per SM a CTA shape reaches, limited by shared memory (228 KB per
// SM, 1 KB reserved per CTA) and the 64-warp / 32-CTA limits.
int warps_per_sm(size_t smem, int block) {
    const size_t per_sm = 233472;
    int by_smem = (int)(per_sm / (smem + 1024));
    int ctas = std::min(std::min(by_smem, 32), 64 / (block / 32));
    return ctas * (block / 32);
}

// Launch configuration: the kernel kind, fold, accumulator, and the block
// size that gives the most resident warps for this histogram size.
FoldConfig choose_config(pf_ctx* ctx, const Job& j, uint32_t max_len, bool& ok) {
    FoldConfig c{};
    c.kind = KIND_FOLD;
    c.cnt16 = false;
    c.algo = j.algo;
    const bool chosen = (j.mode & PF_MODE_CHOSEN) != 0;
    c.fold = chosen ? FOLD_EXACT : FOLD_REF;
    if (j.algo == ALGO_LS) {
        if (chosen) c.fold = (j.mode & PF_FOLD_EXACT) ? FOLD_EXACT : FOLD_DF;
        if (j.mode & PF_FOLD_DF) c.fold = FOLD_DF;
        if (j.mode & PF_FOLD_F32) c.fold = FOLD_F32;
    }
    c.acc = AOVACC_F32;
    c.n_sm = ctx->n_sm;
    c.rounds = 1;
    c.ovl = (j.algo == ALGO_CE) ? (j.po > 1 || j.mo > 1) : (j.algo == ALGO_AOV && j.po > 1);
    if (chosen && !c.ovl && (j.algo == ALGO_CE || j.algo == ALGO_AOV) && max_len < 65536u) {
        c.kind = KIND_BIN;
        c.cnt16 = (j.algo == ALGO_CE);
        c.ref_stats = (j.mode & PF_REF_STATS) != 0;
        // The reference statistic (parity tests) is built in one shape only.
        c.persist = false;
    } else if (j.algo == ALGO_AOV && chosen &&
               (uint64_t)max_len * j.po < (1ull << (64 - kFixCountShift)) - 1ull) {
        c.acc = AOVACC_FIX;
    }
    ok = false;
    int best_warps = 0;
    const int blocks[3] = {256, 128, 64};
    for (int b : blocks) {
        FoldConfig t = c;
        t.block = b;
        const size_t sm = fold_smem(t, j.n_phase, j.n_mag);
        if (sm > ctx->smem_optin) continue;
        const int wps = warps_per_sm(sm, b);
        if (wps > best_warps) {
            best_warps = wps;
            c.block = b;
            ok = true;
        }
    }
    return c;
}

// Bin-edge guard of the bin kernel, in units of 2^-20 of a phase bin: the
// reference's quotient folded / bin_size differs from frac(q') * n by less
// than 2 ulp (f32 divide) + n * 2^-23 (bin width rounding) + n * 2^-25
// (f64 -> f32 rounding of the phase) + 2^-20 (q' = t * RN(1/P) against
// RN(t / P): 2 ulp(q) * n <= 2^-20 while |q| * n < 2^30), plus two units of
// margin.
uint32_t edge_guard(uint32_t n) {
    int cl = 0;
    while ((1u << cl) < n + 1u) cl++;
    const double delta =
        ldexp(1.0, cl - 22) + n * ldexp(1.0, -23) + n * ldexp(1.0, -25) + ldexp(1.0, -20);
    return (uint32_t)ceil(delta * 1048576.0) + 2u;
}

// Work list: for each curve (longest first) and each period derivative,
// tiles of `block` consecutive periods.
void build_work(const Job& j, const Layout& L, int block, WorkItem* w) {
    std::vector<uint32_t> order(j.n_curves);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return L.len[a] > L.len[b]; });
    size_t k = 0;
    for (uint32_t c : order) {
        for (uint32_t d = 0; d < j.n_pdt; d++) {
            for (uint64_t p0 = 0; p0 < j.n_per; p0 += block) {
                w[k].curve = c;
                w[k].pdt = d;
                w[k].p0 = (uint32_t)p0;
                w[k].np = (uint32_t)std::min<uint64_t>(block, j.n_per - p0);
                k++;
            }
        }
    }
}

// Curve order of the persistent kernels' queue: longest first, ties in
// input order (a counting sort on the lengths, or a stable sort when the
// longest curve is very long).
void build_order(const Layout& L, uint64_t n_curves, uint32_t* order) {
    if (L.max_len <= (1u << 20)) {
        std::vector<uint32_t> start((size_t)L.max_len + 2, 0u);
        for (uint64_t c = 0; c < n_curves; c++) start[(size_t)(L.max_len - L.len[c]) + 1]++;
        for (size_t k = 1; k < start.size(); k++) start[k] += start[k - 1];
        for (uint64_t c = 0; c < n_curves; c++) order[start[L.max_len - L.len[c]]++] = (uint32_t)c;
        return;
    }
    std::iota(order, order + n_curves, 0u);
    std::stable_sort(order, order + n_curves,
                     [&](uint32_t a, uint32_t b) { return L.len[a] > L.len[b]; });
}

// Copy one curve into the packed staging area, checking times are finite
// and raising tmax to their largest magnitude.
bool copy_curve(const float* t, const float* m, uint32_t n, float* dt, float* dm, uint32_t pad,
                float& tmax) {
    bool ok = true;
    float mx = tmax;
    for (uint32_t i = 0; i < n; i++) {
        const float x = t[i];
        ok &= std::isfinite(x);
        mx = std::max(mx, std::fabs(x));
        dt[i] = x;
    }
    tmax = mx;
    if (n) memcpy(dm, m, (size_t)n * sizeof(float));
    for (uint32_t i = n; i < pad; i++) {
        dt[i] = 0.0f;
        dm[i] = 0.0f;
    }
    return ok;
}

// Host-side plan: packed layout, launch configuration and the offsets of
// each section in the staging block.  With `with_points` the staging block
// also carries the curve points (host-pointer callers); device callers'
// points are gathered on the device instead.
int plan(pf_ctx* ctx, const Job& j, const uint64_t* lengths, bool with_points, bool with_grid,
         Layout& L, FoldConfig& cfg) {
    L.off.resize(j.n_curves);
    L.len.resize(j.n_curves);
    size_t run = 0;
    for (uint64_t c = 0; c < j.n_curves; c++) {
        if (lengths[c] > 0xFFFFFFFFull)
            return fail(ctx, PF_EINVAL, "curve %llu too long", (unsigned long long)c);
        L.off[c] = (int64_t)run;
        L.len[c] = (uint32_t)lengths[c];
        L.max_len = std::max(L.max_len, L.len[c]);
        run += align_up(lengths[c], 4);
    }
    L.total_pts = run;

    bool ok_cfg = false;
    cfg = choose_config(ctx, j, L.max_len, ok_cfg);
    if (!ok_cfg)
        return fail(ctx, PF_EUNSUPPORTED,
                    "histogram of %u x %u bins does not fit in shared memory", j.n_phase,
                    j.algo == ALGO_CE ? j.n_mag : 1u);
    const uint64_t tiles_per = (j.n_per + cfg.block - 1) / cfg.block;
    const uint64_t n_work64 = j.n_curves * j.n_pdt * tiles_per;
    if (n_work64 > 0x7FFFFFFFull) return fail(ctx, PF_EINVAL, "too much work for one launch");
    L.n_work = (uint32_t)n_work64;

    size_t o = 0;
    L.o_t = o;
    if (with_points) o = align_up(o + L.total_pts * 4, 256);
    L.o_m = o;
    if (with_points) o = align_up(o + L.total_pts * 4, 256);
    L.o_curves = o;
    o = align_up(o + j.n_curves * sizeof(CurveDesc), 256);
    L.o_work = o;
    // Queue kernels take a curve order (the device derives the items);
    // the others a host-built work list.
    if (uses_queue(cfg.kind, cfg.fold))
        o = align_up(o + (size_t)j.n_curves * sizeof(uint32_t), 256);
    else
        o = align_up(o + (size_t)L.n_work * sizeof(WorkItem), 256);
    L.o_periods = o;
    if (with_grid) o = align_up(o + j.n_per * 4, 256);
    L.o_pdts = o;
    if (with_grid) o = align_up(o + j.n_pdt * 4, 256);
    L.o_srcoff = o;
    if (!with_points) o = align_up(o + j.n_curves * 8, 256);
    L.o_tmax = o;
    if (with_points) o = align_up(o + 4, 256);
    L.bytes = o;
    return PF_OK;
}

// Wait until the previous call's copy out of the pinned staging block has
// finished, so the block can be rewritten.
int staging_ready(pf_ctx* ctx) {
    if (ctx->staged_pending) {
        PF_CUDA(cudaEventSynchronize(ctx->ev_staged), "staging event");
        ctx->staged_pending = false;
    }
    return PF_OK;
}

void fill_meta(pf_ctx* ctx, const Job& j, Layout& L, const FoldConfig& cfg, char* hb) {
    CurveDesc* hc = (CurveDesc*)(hb + L.o_curves);
    for (uint64_t c = 0; c < j.n_curves; c++) {
        CurveDesc d{};
        d.off = L.off[c];
        d.n = L.len[c];
        hc[c] = d;
    }
    if (uses_queue(cfg.kind, cfg.fold)) {
        // Item-to-curve map for PF_TIMING is made per class at launch time.
        L.order.resize(j.n_curves);
        build_order(L, j.n_curves, L.order.data());
        memcpy(hb + L.o_work, L.order.data(), j.n_curves * sizeof(uint32_t));
        return;
    }
    WorkItem* w = (WorkItem*)(hb + L.o_work);
    build_work(j, L, cfg.block, w);
    if (j.mode & PF_TIMING) {
        ctx->stamp_curves.resize(L.n_work);
        for (uint32_t k = 0; k < L.n_work; k++) ctx->stamp_curves[k] = w[k].curve;
        ctx->stamp_n_curves = j.n_curves;
    }
}

// Length classes of the queue kernels: [0,64), [64,256), [256,1024),
// [1024,4096), [4096,...).  Each class runs as its own launch with the
// launch shape the autotuner picked for it.
constexpr uint32_t kClassEdges[] = {64, 256, 1024, 4096};
constexpr int kClasses = 5;
int length_class(uint32_t len) {
    int c = 0;
    for (uint32_t e : kClassEdges) c += (len >= e) ? 1 : 0;
    return c;
}
const char* class_name(int c) {
    static const char* names[kClasses] = {"[0,64)", "[64,256)", "[256,1024)", "[1024,4096)",
                                          "[4096,inf)"};
    return names[c];
}
// Queue counters in the context's misc block: one per class, one for tuning.
// (Offset 0 holds max |t|; kFgridZeroOffset a zero period derivative.)
constexpr size_t kCounterOffset = 64;
constexpr size_t kFgridZeroOffset = 48;
// Length classes whose curves fit the shared-histogram kernel's staging
// (kWarpMaxPoints = 1024 points): [0,64), [64,256), [256,1024).
constexpr int kWarpClassMax = 2;
constexpr int kTuneCounter = kClasses;

// Items of a queue launch over n_curves curves, `per_item` periods each.
uint64_t queue_items(const Job& j, uint64_t n_curves, int per_item) {
    return n_curves * j.n_pdt * ((j.n_per + per_item - 1) / per_item);
}

std::string tune_key(const Job& j, const FoldConfig& c, int cls) {
    char b[160];
    snprintf(b, sizeof(b), "%s %s%s%s%s ph=%u mag=%u pdt=%s sem=%s class=%s",
             c.algo == ALGO_CE ? "ce" : c.algo == ALGO_AOV ? "aov" : "ls",
             c.kind == KIND_BIN ? "bin" : (c.fold == FOLD_DF ? "fold-split" : "fold-exact"),
             c.cnt16 ? "-cnt16" : "", c.ref_stats ? "-refstats" : "",
             j.fgrid ? ((j.mode & PF_TRIG_SINCOS) ? "-fgrid-sincos"
                        : (j.mode & PF_TRIG_RECURRENCE) ? "-fgrid-recurrence" : "-fgrid")
                     : (j.mode & PF_BINS_SHARED) ? "-shared-bins" : "",
             j.n_phase, c.algo == ALGO_CE ? j.n_mag : 0u, j.n_pdt > 1 ? "many" : "one",
             use_cpu_semantics(j.mode) ? "cpu" : "cuda", class_name(cls));
    return b;
}

cudaError_t launch_fold_sem(const Job& j, const FoldConfig& c, const FoldParams& p,
                            uint32_t n_work, cudaStream_t s) {
    return use_cpu_semantics(j.mode) ? launch_fold_cpusem(c, p, n_work, s)
                                     : launch_fold_cudasem(c, p, n_work, s);
}

// Launch shape of one length class.  Cached per context; the first time a
// key is met, every candidate (block 64 / 128 / 256 where shared memory
// allows, persistent or one CTA per item) is timed with CUDA events on a
// sample of the class (a contiguous run of its curves from the middle of
// the class, about 2e9 point evaluations) and the fastest kept.  The sample
// writes cells of the real output, which the class launch rewrites.  Every
// candidate computes the same values; only the time differs.  No tuning
// (the base shape) with PF_NO_TUNE or while the stream is being captured.
int tuned_config(pf_ctx* ctx, const Job& j, const FoldConfig& base, int cls, uint64_t c0,
                 uint64_t nc, uint64_t cls_points, const FoldParams& p, cudaStream_t s,
                 FoldConfig& out) {
    out = base;
    // LS on a uniform frequency grid: the trig form is a candidate axis too
    // (MUFU sin / cos per evaluation, or the recurrence along the grid with
    // 4 or 8 frequencies per thread); PF_TRIG_* keeps one form.
    const bool rec_ok = j.fgrid && base.algo == ALGO_LS && base.fold == FOLD_DF;
    const bool only_rec = rec_ok && (j.mode & PF_TRIG_RECURRENCE);
    const bool no_rec = !rec_ok || (j.mode & PF_TRIG_SINCOS);
    // Likewise the binning strategy of the chosen CE / AOV kernels:
    // per-thread privatised histograms, or shared histograms with atomics
    // (PF_BINS_SHARED keeps the latter where the curves fit it).
    const bool warp_ok = base.kind == KIND_BIN && !base.ref_stats && cls <= kWarpClassMax;
    const bool only_warp = warp_ok && (j.mode & PF_BINS_SHARED);
    if (only_rec) {
        out.kind = KIND_LSREC;
        out.block = 256;
        out.rounds = 8;
        out.persist = false;
    }
    if (only_warp) {
        out.kind = KIND_BINWARP;
        out.block = 256;
        out.rounds = 1;
        out.persist = false;
    }
    const std::string key = tune_key(j, base, cls);
    auto it = ctx->tuned.find(key);
    if (it != ctx->tuned.end()) {
        out.kind = it->second.kind;
        out.block = it->second.block;
        out.persist = it->second.persist;
        out.rounds = it->second.rounds;
        return PF_OK;
    }
    if (j.mode & PF_NO_TUNE) return PF_OK;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    PF_CUDA(cudaStreamIsCapturing(s, &cap), "capture query");
    if (cap != cudaStreamCaptureStatusNone) return PF_OK;

    const double per_curve = (double)cls_points / (double)nc * (double)j.n_per * (double)j.n_pdt;
    uint64_t k = (uint64_t)std::max(1.0, std::ceil(2e9 / std::max(per_curve, 1.0)));
    // Enough curves that the candidate with the largest items (2048 periods)
    // still has four items per SM: a sample that leaves SMs idle would
    // favour small items over what the whole class runs best with.
    const uint64_t big_items = j.n_pdt * ((j.n_per + 2047) / 2048);
    k = std::max<uint64_t>(k, (4ull * (uint64_t)std::max(ctx->n_sm, 1) + big_items - 1) /
                                  std::max<uint64_t>(big_items, 1));
    k = std::min(k, nc);
    const uint64_t s0 = c0 + (nc - k) / 2;
    FoldParams ps = p;
    ps.stamps = nullptr;
    ps.bins = nullptr;
    ps.q.order = p.q.order + s0;
    ps.q.next = reinterpret_cast<unsigned*>((char*)ctx->d_misc.p + kCounterOffset) + kTuneCounter;
    pf_ctx::Tuned best{out.kind, out.block, out.persist, out.rounds, 1e30f, 0.0f, 0};
    // Candidates: block x persistent-or-not, and for the bin kernel 1 or 4
    // rounds of periods per item; for the recurrence 4 or 8 frequencies per
    // thread.  The reference statistic is built in one shape only.
    std::vector<FoldConfig> cands;
    const bool shapes = !(base.kind == KIND_BIN && base.ref_stats);
    if (!only_rec && !only_warp) {
        for (int block : {64, 128, 256}) {
            FoldConfig t = base;
            t.block = block;
            if (fold_smem(t, j.n_phase, j.n_mag) > ctx->smem_optin) continue;
            for (int shape = 0; shape < (shapes ? 4 : 1); shape++) {
                t.persist = (shape & 1) != 0;
                t.rounds = (base.kind == KIND_BIN && (shape & 2)) ? 4 : 1;
                if (base.kind != KIND_BIN && (shape & 2)) continue;
                cands.push_back(t);
            }
        }
    }
    // The shared-histogram binning (one histogram per warp and period,
    // shared atomics) for classes of curves shorter than its staging limit.
    if (warp_ok) {
        for (int block : {128, 256})
            for (int persist = 0; persist < 2; persist++) {
                FoldConfig t = base;
                t.kind = KIND_BINWARP;
                t.block = block;
                t.rounds = 1;
                t.persist = persist != 0;
                if (fold_smem(t, j.n_phase, j.n_mag) <= ctx->smem_optin) cands.push_back(t);
            }
    }
    if (!no_rec) {
        for (int block : {128, 256})
            for (int r : {4, 8})
                for (int persist = 0; persist < 2; persist++) {
                    FoldConfig t = base;
                    t.kind = KIND_LSREC;
                    t.block = block;
                    t.rounds = r;
                    t.persist = persist != 0;
                    cands.push_back(t);
                }
    }
    // Fastest of `reps` timed launches of candidate t on the sample.
    auto time_cand = [&](const FoldConfig& t, int reps, float& ms) -> int {
        const uint64_t nw = queue_items(j, k, item_periods(t));
        ps.q.n_work = (uint32_t)nw;
        for (int rep = 0; rep < reps; rep++) {
            float m = 0.0f;
            PF_CUDA(cudaEventRecord(ctx->ev0, s), "event");
            PF_CUDA(launch_fold_sem(j, t, ps, (uint32_t)nw, s), "tuning launch");
            PF_CUDA(cudaEventRecord(ctx->ev1, s), "event");
            PF_CUDA(cudaEventSynchronize(ctx->ev1), "tuning sync");
            PF_CUDA(cudaEventElapsedTime(&m, ctx->ev0, ctx->ev1), "event time");
            ms = std::min(ms, m);
        }
        ctx->launches += (uint64_t)reps;
        return PF_OK;
    };
    // First pass: a warm-up launch, then the faster of two.
    std::vector<std::pair<FoldConfig, float>> timed;
    for (const FoldConfig& t : cands) {
        const uint64_t nw = queue_items(j, k, item_periods(t));
        if (nw == 0 || nw > 0x7FFFFFFFull) continue;
        float warm = 1e30f, ms = 1e30f;
        int rc;
        if ((rc = time_cand(t, 1, warm)) != PF_OK || (rc = time_cand(t, 2, ms)) != PF_OK)
            return rc;
        timed.emplace_back(t, ms);
        best.candidates++;
        best.ms_worst = std::max(best.ms_worst, ms);
    }
    if (best.candidates == 0) return PF_OK;
    // Second pass over the candidates within 6% of the fastest: shapes that
    // close differ by less than the launch-to-launch spread of a ~1 ms
    // sample, so they are timed again, in turns (round robin, so that a
    // drift of the clock or of L2 state falls on all of them alike), and the
    // fastest launch of either pass decides.
    float first = 1e30f;
    for (const auto& c : timed) first = std::min(first, c.second);
    std::vector<size_t> close;
    for (size_t i = 0; i < timed.size(); i++)
        if (timed[i].second <= 1.06f * first) close.push_back(i);
    if (close.size() > 1)
        for (int round = 0; round < 3; round++)
            for (size_t i : close) {
                int rc;
                if ((rc = time_cand(timed[i].first, 1, timed[i].second)) != PF_OK) return rc;
            }
    for (const auto& c : timed) {
        if (c.second < best.ms) {
            best.ms = c.second;
            best.kind = c.first.kind;
            best.block = c.first.block;
            best.persist = c.first.persist;
            best.rounds = c.first.rounds;
        }
    }
    ctx->tuned[key] = best;
    out.kind = best.kind;
    out.block = best.block;
    out.persist = best.persist;
    out.rounds = best.rounds;
    return PF_OK;
}

// One launch per length class of a queue kernel (curves longest first, so
// each class is a contiguous run of the order array), after tuning.
int launch_classes(pf_ctx* ctx, const Job& j, const Layout& L, const FoldConfig& cfg,
                   const FoldParams& p, cudaStream_t s) {
    struct Range {
        uint64_t c0, n, points;
    };
    Range r[kClasses] = {};
    bool seen[kClasses] = {};
    for (uint64_t i = 0; i < j.n_curves; i++) {
        const int c = length_class(L.len[L.order[i]]);
        if (!seen[c]) {
            seen[c] = true;
            r[c].c0 = i;
        }
        r[c].n++;
        r[c].points += L.len[L.order[i]];
    }
    FoldConfig cc[kClasses];
    uint64_t total_items = 0;
    int rc;
    for (int c = 0; c < kClasses; c++) {
        if (!r[c].n) continue;
        if ((rc = tuned_config(ctx, j, cfg, c, r[c].c0, r[c].n, r[c].points, p, s, cc[c])) !=
            PF_OK)
            return rc;
        total_items += queue_items(j, r[c].n, item_periods(cc[c]));
    }
    if (j.mode & PF_ONE_LAUNCH) {
        // Every curve in one launch with the shape tuned for the class that
        // holds the most points (or, where that shape is the shared-histogram
        // binning and longer curves are present, the longest class's).
        int d = -1, longest = -1;
        for (int c = 0; c < kClasses; c++) {
            if (!r[c].n) continue;
            if (d < 0 || r[c].points > r[d].points) d = c;
            longest = c;
        }
        if (cc[d].kind == KIND_BINWARP && longest > kWarpClassMax) d = longest;
        const FoldConfig one = cc[d];
        const uint64_t pts = L.total_pts;
        for (int c = 0; c < kClasses; c++) r[c] = Range{0, 0, 0};
        r[0] = Range{0, j.n_curves, pts};
        cc[0] = one;
        total_items = queue_items(j, j.n_curves, item_periods(one));
    }
    if (total_items > 0x7FFFFFFFull) return fail(ctx, PF_EINVAL, "too much work for one launch");
    if (j.mode & PF_TIMING) {
        if ((rc = ensure_dev(ctx, ctx->d_stamps, (size_t)total_items * 16)) != PF_OK) return rc;
        PF_CUDA(cudaMemsetAsync(ctx->d_stamps.p, 0, (size_t)total_items * 16, s), "memset");
        ctx->stamp_curves.resize(total_items);
        ctx->stamp_n_curves = j.n_curves;
        ctx->stamp_stream = s;
    }
    PF_CUDA(cudaEventRecord(ctx->ev0, s), "event");
    uint64_t base = 0;
    for (int c = 0; c < kClasses; c++) {
        if (!r[c].n) continue;
        const uint64_t nw = queue_items(j, r[c].n, item_periods(cc[c]));
        FoldParams pc = p;
        pc.q.order = p.q.order + r[c].c0;
        pc.q.n_work = (uint32_t)nw;
        pc.q.next = reinterpret_cast<unsigned*>((char*)ctx->d_misc.p + kCounterOffset) + c;
        pc.stamps = nullptr;
        if (j.mode & PF_TIMING) {
            pc.stamps = (unsigned long long*)ctx->d_stamps.p + 2 * base;
            const uint64_t tpc = queue_items(j, 1, item_periods(cc[c]));
            for (uint64_t k = 0; k < nw; k++)
                ctx->stamp_curves[base + k] = L.order[r[c].c0 + k / tpc];
        }
        PF_CUDA(launch_fold_sem(j, cc[c], pc, (uint32_t)nw, s), "fold kernel launch");
        ctx->launches++;
        base += nw;
    }
    PF_CUDA(cudaEventRecord(ctx->ev1, s), "event");
    ctx->timed_pending = true;
    return PF_OK;
}

// Device pipeline shared by both entry styles: preparation kernel, fused
// kernel, optional peak search.  `p` has the input pointers set.
int device_pipeline(pf_ctx* ctx, const Job& j, const Layout& L, const FoldConfig& cfg,
                    FoldParams& p, CurveDesc* dcurves, float* d_out, cudaStream_t s,
                    const unsigned* d_tmax_staged = nullptr) {
    const bool cpu = use_cpu_semantics(j.mode);
    p.n_per = (uint32_t)j.n_per;
    p.n_pdt = (uint32_t)j.n_pdt;
    p.n_phase = j.n_phase;
    p.n_mag = j.n_mag;
    p.p_overlap = j.po;
    p.m_overlap = j.mo;
    p.phase_bin_size = bin_size(j.n_phase, cpu);
    p.mag_bin_size = bin_size(j.n_mag, cpu);
    p.out = d_out;
    p.edge_d = edge_guard(j.n_phase);
    p.fgrid = j.fgrid ? 1 : 0;
    p.f0 = j.f0;
    p.df = j.df;
    const uint32_t ncur = (uint32_t)j.n_curves;
    int rc;
    if ((rc = ensure_dev(ctx, ctx->d_misc, 256)) != PF_OK) return rc;
    static_assert(kCounterOffset + 4 * (kClasses + 1) <= 256, "counters fit the misc block");
    Stage stage_prep("pf prepare");
    if (d_tmax_staged) {
        // Host-packed inputs: max |t| came with them.
        p.tmax_bits = d_tmax_staged;
    } else {
        p.tmax_bits = (const unsigned*)ctx->d_misc.p;
        PF_CUDA(launch_tmax(p.t, L.total_pts, (unsigned*)ctx->d_misc.p, s), "max|t| kernel");
        ctx->launches++;
    }
    if (cfg.kind == KIND_BIN && j.algo == ALGO_CE) {
        if ((rc = ensure_dev(ctx, ctx->d_aux64, L.total_pts * 8 + 32)) != PF_OK) return rc;
        p.aux64 = (const uint64_t*)ctx->d_aux64.p;
        cudaError_t e = cpu ? launch_binaux_cpusem(p.m, ctx->d_aux64.p, dcurves, ncur, j.n_mag,
                                                   p.mag_bin_size, cfg.block, cfg.cnt16, s)
                            : launch_binaux_cudasem(p.m, ctx->d_aux64.p, dcurves, ncur,
                                                    j.n_mag, p.mag_bin_size, cfg.block,
                                                    cfg.cnt16, s);
        PF_CUDA(e, "CE bin preparation kernel");
        ctx->launches++;
    } else if (cfg.kind == KIND_BIN && j.algo == ALGO_AOV) {
        if ((rc = ensure_dev(ctx, ctx->d_aux32, L.total_pts * 4 + 16)) != PF_OK) return rc;
        p.aux32 = (const uint32_t*)ctx->d_aux32.p;
        PF_CUDA(launch_aov_fix32_prep(p.m, (uint32_t*)ctx->d_aux32.p, dcurves, ncur, s),
                "AOV fixed-point preparation kernel");
        ctx->launches++;
    } else if (j.algo == ALGO_CE) {
        if ((rc = ensure_dev(ctx, ctx->d_aux32, L.total_pts * 4 + 16)) != PF_OK) return rc;
        p.aux32 = (const uint32_t*)ctx->d_aux32.p;
        const int flag_sat = j.mo > 1 ? 1 : 0;
        cudaError_t e = cpu ? launch_magbin_cpusem(p.m, (uint32_t*)ctx->d_aux32.p, dcurves, ncur,
                                                   j.n_mag, p.mag_bin_size, flag_sat, s)
                            : launch_magbin_cudasem(p.m, (uint32_t*)ctx->d_aux32.p, dcurves,
                                                    ncur, j.n_mag, p.mag_bin_size, flag_sat, s);
        PF_CUDA(e, "magnitude-bin kernel");
        ctx->launches++;
    } else if (j.algo == ALGO_AOV) {
        if (cfg.acc == AOVACC_FIX) {
            if ((rc = ensure_dev(ctx, ctx->d_aux64, L.total_pts * 8 + 32)) != PF_OK) return rc;
            p.aux64 = (const uint64_t*)ctx->d_aux64.p;
            PF_CUDA(launch_aov_fix_prep(p.m, (uint64_t*)ctx->d_aux64.p, dcurves, ncur, j.po, s),
                    "AOV fixed-point preparation kernel");
        } else {
            PF_CUDA(launch_aov_mean(p.m, dcurves, ncur, s), "AOV mean kernel");
        }
        ctx->launches++;
    }
    p.stamps = nullptr;
    Stage stage_fold(j.algo == ALGO_LS ? "pf LS fold" : j.algo == ALGO_CE ? "pf CE bins"
                                                                          : "pf AOV bins");
    if (uses_queue(cfg.kind, cfg.fold)) {
        // The staged work section holds the curve order (fill_meta).
        p.q.order = reinterpret_cast<const uint32_t*>(p.work);
        p.work = nullptr;
        if ((rc = launch_classes(ctx, j, L, cfg, p, s)) != PF_OK) return rc;
    } else {
        if (j.mode & PF_TIMING) {
            if ((rc = ensure_dev(ctx, ctx->d_stamps, (size_t)L.n_work * 16)) != PF_OK) return rc;
            PF_CUDA(cudaMemsetAsync(ctx->d_stamps.p, 0, (size_t)L.n_work * 16, s), "memset");
            p.stamps = (unsigned long long*)ctx->d_stamps.p;
            ctx->stamp_stream = s;
        }
        PF_CUDA(cudaEventRecord(ctx->ev0, s), "event");
        PF_CUDA(launch_fold_sem(j, cfg, p, L.n_work, s), "fold kernel launch");
        ctx->launches++;
        PF_CUDA(cudaEventRecord(ctx->ev1, s), "event");
        ctx->timed_pending = true;
    }
    if (j.stats) {
        // One block: [curve][mean, std, median, mad], then the best cells'
        // indices and values, so the results come back in one copy.
        Stage stage_stats("pf statistics");
        const size_t pk = (size_t)j.n_curves * std::max<uint32_t>(j.n_top, 1u);
        const size_t b_st = (size_t)j.n_curves * 16;
        if ((rc = ensure_dev(ctx, ctx->d_stat, b_st + pk * 12)) != PF_OK) return rc;
        char* st = (char*)ctx->d_stat.p;
        PF_CUDA(launch_stats(d_out, j.n_curves, (uint32_t)(j.n_per * j.n_pdt),
                             j.algo == ALGO_CE ? 0 : 1, j.n_top, (float*)st,
                             (int64_t*)(st + b_st), (float*)(st + b_st + pk * 8), s),
                "statistics kernel launch");
        ctx->launches++;
    }
    if (j.peaks && j.n_peaks > 0) {
        Stage stage_peaks("pf peak search");
        const size_t pk = (size_t)j.n_curves * j.n_peaks;
        if ((rc = ensure_dev(ctx, ctx->d_pidx, pk * 8)) != PF_OK) return rc;
        if ((rc = ensure_dev(ctx, ctx->d_pval, pk * 4)) != PF_OK) return rc;
        const int use_max = (j.algo == ALGO_CE) ? 0 : 1;
        PF_CUDA(launch_peaks(d_out, j.n_curves, j.n_per * j.n_pdt, j.n_peaks, j.min_distance,
                             use_max, (int64_t*)ctx->d_pidx.p, (float*)ctx->d_pval.p, s),
                "peak kernel launch");
        ctx->launches++;
    }
    return PF_OK;
}

void read_kernel_time(pf_ctx* ctx) {
    if (!ctx->timed_pending) return;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) ctx->last_ms = ms;
    else cudaGetLastError();
    ctx->timed_pending = false;
}

// Register a PF_ASYNC call for pf_wait: its peaks (n entries) sit in the
// next pending slot's pinned block once the slot's event has completed.
int push_pending(pf_ctx* ctx, const Job& j, size_t n, bool work, cudaStream_t s) {
    pf_ctx::Pending& q = ctx->pend[(ctx->pend_head + ctx->pend_count) % pf_ctx::kMaxPending];
    q.out_idx = j.out_idx;
    q.out_val = j.out_val;
    q.n = n;
    q.work = work;
    if (work) PF_CUDA(cudaEventRecord(q.done, s), "event");
    ctx->pend_count++;
    return PF_OK;
}

// Queue the device-to-host copy of a small result into the pinned result
// block at byte offset `at` (the block must already hold it), and its copy
// on into the caller's array once the call has synchronised.
int queue_result(pf_ctx* ctx, void* dst, const void* d_src, size_t n, size_t at,
                 cudaStream_t s) {
    char* h = (char*)ctx->h_res.p + at;
    PF_CUDA(cudaMemcpyAsync(h, d_src, n, cudaMemcpyDeviceToHost, s), "D2H results");
    ctx->res_copies.push_back(pf_ctx::HostCopy{dst, h, n});
    return PF_OK;
}

// End of a synchronous host call: mark the call's end, wait for it, hand
// the queued small results to the caller.
int finish_sync(pf_ctx* ctx, cudaStream_t s) {
    int rc;
    if ((rc = mark_done(ctx, s)) != PF_OK) return rc;
    PF_CUDA(cudaStreamSynchronize(s), "stream synchronize");
    ctx->staged_pending = false;
    for (const pf_ctx::HostCopy& c : ctx->res_copies) memcpy(c.dst, c.src, c.n);
    ctx->res_copies.clear();
    read_kernel_time(ctx);
    return PF_OK;
}

// Copy a peak call's results (d_pidx / d_pval, n_curves x n_peaks) back:
// into the caller's arrays, or with PF_ASYNC into the next pending slot's
// pinned block (free: its last user was collected, so no copy into it is
// in flight) and register the call for pf_wait.
int copy_peaks_back(pf_ctx* ctx, const Job& j, bool async, cudaStream_t s) {
    const size_t pk = (size_t)j.n_curves * j.n_peaks;
    void* hi = j.out_idx;
    void* hv = j.out_val;
    if (async && pk > 0) {
        pf_ctx::Pending& q = ctx->pend[(ctx->pend_head + ctx->pend_count) % pf_ctx::kMaxPending];
        const int rc = ensure_pinned(ctx, q.res, pk * 12);
        if (rc != PF_OK) return rc;
        hi = q.res.p;
        hv = (char*)q.res.p + pk * 8;
    }
    if (pk > 0 && !async) {
        // Through the pinned result block; the caller's arrays are filled
        // after the synchronisation.
        int rc = ensure_pinned(ctx, ctx->h_res, pk * 12);
        if (rc != PF_OK) return rc;
        if ((rc = queue_result(ctx, hi, ctx->d_pidx.p, pk * 8, 0, s)) != PF_OK) return rc;
        return queue_result(ctx, hv, ctx->d_pval.p, pk * 4, pk * 8, s);
    }
    if (pk > 0) {
        PF_CUDA(cudaMemcpyAsync(hi, ctx->d_pidx.p, pk * 8, cudaMemcpyDeviceToHost, s),
                "D2H peak indices");
        PF_CUDA(cudaMemcpyAsync(hv, ctx->d_pval.p, pk * 4, cudaMemcpyDeviceToHost, s),
                "D2H peak values");
    }
    return async ? push_pending(ctx, j, pk, true, s) : PF_OK;
}

// The whole pipeline for host-pointer inputs.
int run_host(pf_ctx* ctx, const Job& j, const float* const* times, const float* const* mags,
             const uint64_t* lengths) {
    ctx->res_copies.clear();
    int rc = validate_common(ctx, j);
    if (rc != PF_OK) return rc;
    const bool async = (j.mode & PF_ASYNC) != 0;
    if (async) {
        if (!j.peaks) return fail(ctx, PF_EINVAL, "PF_ASYNC applies to the peak calls only");
        if (j.mode & PF_TIMING) return fail(ctx, PF_EINVAL, "PF_ASYNC excludes PF_TIMING");
        if (ctx->pend_count == pf_ctx::kMaxPending)
            return fail(ctx, PF_EINVAL, "%d PF_ASYNC calls are pending; collect one with pf_wait",
                        pf_ctx::kMaxPending);
    }
    if ((j.mode & PF_HOST_NORMALIZE) && (j.mode & PF_HOST_CENTER))
        return fail(ctx, PF_EINVAL, "PF_HOST_NORMALIZE and PF_HOST_CENTER exclude each other");
    if (j.n_curves == 0) return async ? push_pending(ctx, j, 0, false, nullptr) : PF_OK;
    if (!times || !mags || !lengths) return fail(ctx, PF_EINVAL, "times/mags/lengths is NULL");
    const uint64_t n_cells = j.n_per * j.n_pdt;
    if (n_cells == 0) return async ? push_pending(ctx, j, 0, false, nullptr) : PF_OK;
    if ((rc = check_grid_host(ctx, j)) != PF_OK) return rc;
    for (uint64_t c = 0; c < j.n_curves; c++)
        if (lengths[c] > 0 && (!times[c] || !mags[c]))
            return fail(ctx, PF_EINVAL, "curve %llu has a NULL array", (unsigned long long)c);
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");

    Layout L;
    FoldConfig cfg;
    if ((rc = plan(ctx, j, lengths, true, true, L, cfg)) != PF_OK) return rc;
    if ((rc = staging_ready(ctx)) != PF_OK) return rc;
    if ((rc = ensure_pinned(ctx, ctx->h_in, L.bytes)) != PF_OK) return rc;
    const int slot = ctx->in_slot;
    DevBuf& din = slot ? ctx->d_in2 : ctx->d_in;
    if ((rc = ensure_dev(ctx, din, L.bytes)) != PF_OK) return rc;
    char* hb = (char*)ctx->h_in.p;
    float* ht = (float*)(hb + L.o_t);
    float* hm = (float*)(hb + L.o_m);

    // Pack the curves (several host threads for large batches).
    {
        Stage stage_pack("pf pack");
        const CurveTasks T = curve_tasks(L.off, L.total_pts);
        std::vector<int> bad(T.count(), 0);
        std::vector<float> tmx(T.count(), 0.0f);
        auto worker = [&](unsigned w) {
            for (uint64_t c = T.first[w]; c < T.first[w + 1]; c++) {
                const uint32_t n = L.len[c];
                const uint32_t pad = (uint32_t)align_up(n, 4);
                if (!copy_curve(times[c], mags[c], n, ht + L.off[c], hm + L.off[c], pad, tmx[w]))
                    bad[w] = 1;
                // Magnitude preparation fused into the packing (numpy's
                // values, as pf_normalize_mags / pf_center_mags).
                if (n && (j.mode & PF_HOST_NORMALIZE))
                    normalize_curve(hm + L.off[c], n, hm + L.off[c]);
                else if (n && (j.mode & PF_HOST_CENTER))
                    center_curve(hm + L.off[c], n, hm + L.off[c]);
            }
        };
        ctx->pool.run(T.count(), T.width, worker);
        for (int b : bad)
            if (b) return fail(ctx, PF_EINVAL, "times must be finite");
        // The kernels' range guard reads max |t| as float bits: found while
        // packing, so no reduction kernel is needed.
        float tmax = 0.0f;
        for (float x : tmx) tmax = std::max(tmax, x);
        memcpy(hb + L.o_tmax, &tmax, 4);
    }
    fill_meta(ctx, j, L, cfg, hb);
    if (!j.fgrid) memcpy(hb + L.o_periods, j.periods, j.n_per * 4);
    memcpy(hb + L.o_pdts, j.pdts, j.n_pdt * 4);

    cudaStream_t s = ctx->stream;
    char* db = (char*)din.p;
    if ((rc = order_after_previous(ctx, s)) != PF_OK) return rc;
    // The copy waits only for the kernels that last read this input block
    // (two host calls back), not for the previous call, whose kernels it
    // overlaps; the kernels of this call wait for the copy.
    CallEnd call_end{ctx, s};
    {
        Stage stage_h2d("pf H2D");
        PF_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_in_free[slot], 0), "stream wait");
        PF_CUDA(cudaMemcpyAsync(db, hb, L.bytes, cudaMemcpyHostToDevice, ctx->copy_stream),
                "H2D inputs");
        PF_CUDA(cudaEventRecord(ctx->ev_copied[slot], ctx->copy_stream), "event");
    }
    PF_CUDA(cudaEventRecord(ctx->ev_staged, ctx->copy_stream), "event");
    ctx->staged_pending = true;
    ctx->in_slot = slot ^ 1;
    PF_CUDA(cudaStreamWaitEvent(s, ctx->ev_copied[slot], 0), "stream wait");

    FoldParams p{};
    p.t = (const float*)(db + L.o_t);
    p.m = (const float*)(db + L.o_m);
    p.curves = (const CurveDesc*)(db + L.o_curves);
    p.work = (const WorkItem*)(db + L.o_work);
    p.periods = (const float*)(db + L.o_periods);
    p.pdts = (const float*)(db + L.o_pdts);
    const size_t out_bytes = (size_t)j.n_curves * n_cells * 4;
    if ((rc = ensure_dev(ctx, ctx->d_out, out_bytes)) != PF_OK) return rc;
    const size_t bins_bytes = j.out_bins ? out_bytes * bins_per_cell(j) : 0;
    if (j.out_bins) {
        if ((rc = ensure_dev(ctx, ctx->d_bins, bins_bytes)) != PF_OK) return rc;
        PF_CUDA(cudaMemsetAsync(ctx->d_bins.p, 0, bins_bytes, s), "memset");
        p.bins = (uint32_t*)ctx->d_bins.p;
    }
    rc = device_pipeline(ctx, j, L, cfg, p, (CurveDesc*)(db + L.o_curves), (float*)ctx->d_out.p,
                         s, (const unsigned*)(db + L.o_tmax));
    if (rc != PF_OK) return rc;
    if (j.out_bins)
        PF_CUDA(cudaMemcpyAsync(j.out_bins, ctx->d_bins.p, bins_bytes, cudaMemcpyDeviceToHost, s),
                "D2H bin counts");
    if (j.stats) {
        // Through the pinned result block (filled into the caller's arrays
        // after the synchronisation).
        const size_t b_st = (size_t)j.n_curves * 16;
        const size_t pk = (size_t)j.n_curves * j.n_top;
        const size_t pk1 = (size_t)j.n_curves * std::max<uint32_t>(j.n_top, 1u);  // layout
        const size_t bytes = pk > 0 ? b_st + pk1 * 12 : b_st;
        if ((rc = ensure_pinned(ctx, ctx->h_res, bytes)) != PF_OK) return rc;
        char* hr = (char*)ctx->h_res.p;
        PF_CUDA(cudaMemcpyAsync(hr, ctx->d_stat.p, bytes, cudaMemcpyDeviceToHost, s),
                "D2H statistics");
        ctx->res_copies.push_back(pf_ctx::HostCopy{j.out_stats, hr, b_st});
        if (pk > 0) {
            ctx->res_copies.push_back(pf_ctx::HostCopy{j.out_idx, hr + b_st, pk * 8});
            ctx->res_copies.push_back(pf_ctx::HostCopy{j.out_val, hr + b_st + pk1 * 8, pk * 4});
        }
    } else if (!j.peaks) {
        PF_CUDA(cudaMemcpyAsync(j.out, ctx->d_out.p, out_bytes, cudaMemcpyDeviceToHost, s),
                "D2H periodogram");
    } else {
        if ((rc = copy_peaks_back(ctx, j, async, s)) != PF_OK) return rc;
        // PF_ASYNC: the call returns with its work queued.  The staging
        // block stays marked in use until the H2D copy above has finished.
        if (async) {
            ctx->cur_slot = slot;
            call_end.armed = false;
            return mark_done(ctx, s);
        }
    }
    ctx->cur_slot = slot;
    call_end.armed = false;
    return finish_sync(ctx, s);
}

// Device-pointer inputs and output, enqueued on the caller's stream.
int run_dev(pf_ctx* ctx, const Job& j, const float* d_times, const float* d_mags,
            const int64_t* offsets, void* stream_v) {
    int rc = validate_common(ctx, j);
    if (rc != PF_OK) return rc;
    if (j.n_curves == 0) return PF_OK;
    if (!offsets) return fail(ctx, PF_EINVAL, "offsets is NULL");
    const uint64_t n_cells = j.n_per * j.n_pdt;
    if (n_cells == 0) return PF_OK;
    std::vector<uint64_t> lengths(j.n_curves);
    for (uint64_t c = 0; c < j.n_curves; c++) {
        if (offsets[c + 1] < offsets[c] || offsets[c] < 0)
            return fail(ctx, PF_EINVAL, "offsets must be non-decreasing and non-negative");
        lengths[c] = (uint64_t)(offsets[c + 1] - offsets[c]);
    }
    if (offsets[j.n_curves] > 0 && (!d_times || !d_mags))
        return fail(ctx, PF_EINVAL, "d_times/d_mags is NULL");
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    // NULL is the CUDA default stream, as for any CUDA API taking a stream.
    cudaStream_t s = (cudaStream_t)stream_v;

    Layout L;
    FoldConfig cfg;
    if ((rc = plan(ctx, j, lengths.data(), false, false, L, cfg)) != PF_OK) return rc;
    if ((rc = staging_ready(ctx)) != PF_OK) return rc;
    if ((rc = ensure_pinned(ctx, ctx->h_in, L.bytes)) != PF_OK) return rc;
    if ((rc = ensure_dev(ctx, ctx->d_in, L.bytes)) != PF_OK) return rc;
    if ((rc = ensure_dev(ctx, ctx->d_pack, L.total_pts * 8 + 64)) != PF_OK) return rc;
    char* hb = (char*)ctx->h_in.p;
    fill_meta(ctx, j, L, cfg, hb);
    memcpy(hb + L.o_srcoff, offsets, j.n_curves * 8);

    // Order this call after the previous one on this context (its buffers
    // are reused), whichever stream that one ran on.
    if ((rc = order_after_previous(ctx, s)) != PF_OK) return rc;
    char* db = (char*)ctx->d_in.p;
    PF_CUDA(cudaMemcpyAsync(db, hb, L.bytes, cudaMemcpyHostToDevice, s), "H2D metadata");
    PF_CUDA(cudaEventRecord(ctx->ev_staged, s), "event");
    ctx->staged_pending = true;

    float* pt = (float*)ctx->d_pack.p;
    float* pm = pt + L.total_pts;
    CurveDesc* dcurves = (CurveDesc*)(db + L.o_curves);
    PF_CUDA(launch_pack(d_times, d_mags, (const int64_t*)(db + L.o_srcoff), dcurves,
                        (uint32_t)j.n_curves, pt, pm, s),
            "pack kernel");
    ctx->launches++;
    FoldParams p{};
    p.t = pt;
    p.m = pm;
    p.curves = dcurves;
    p.work = (const WorkItem*)(db + L.o_work);
    p.periods = j.periods;
    p.pdts = j.pdts;
    if (j.fgrid) {
        // The one period derivative (0) of a frequency grid, on the device.
        if ((rc = ensure_dev(ctx, ctx->d_misc, 256)) != PF_OK) return rc;
        float* zero = (float*)((char*)ctx->d_misc.p + kFgridZeroOffset);
        PF_CUDA(cudaMemsetAsync(zero, 0, sizeof(float), s), "memset");
        p.pdts = zero;
    }
    rc = device_pipeline(ctx, j, L, cfg, p, dcurves, j.out, s);
    if (rc != PF_OK) return rc;
    return mark_done(ctx, s);
}

// Copy a host CSR offsets array into the context's device metadata block,
// ordered after the previous device-pointer call on this context, on stream
// s.  Returns the device copy and the longest curve.
int stage_offsets(pf_ctx* ctx, const int64_t* offsets, uint64_t n_curves, cudaStream_t s,
                  const int64_t** d_off, uint32_t* max_len) {
    if (!offsets) return fail(ctx, PF_EINVAL, "offsets is NULL");
    uint64_t mx = 0;
    for (uint64_t c = 0; c < n_curves; c++) {
        if (offsets[c + 1] < offsets[c] || offsets[c] < 0)
            return fail(ctx, PF_EINVAL, "offsets must be non-decreasing and non-negative");
        mx = std::max(mx, (uint64_t)(offsets[c + 1] - offsets[c]));
    }
    if (mx > 0xFFFFFFFFull) return fail(ctx, PF_EINVAL, "a curve has more than 2^32-1 points");
    const size_t bytes = (size_t)(n_curves + 1) * 8;
    int rc;
    if ((rc = staging_ready(ctx)) != PF_OK) return rc;
    if ((rc = ensure_pinned(ctx, ctx->h_in, bytes)) != PF_OK) return rc;
    if (ctx->done_recorded) PF_CUDA(cudaStreamWaitEvent(s, ctx->ev_done, 0), "stream wait");
    if ((rc = ensure_dev(ctx, ctx->d_in, bytes)) != PF_OK) return rc;
    memcpy(ctx->h_in.p, offsets, bytes);
    PF_CUDA(cudaMemcpyAsync(ctx->d_in.p, ctx->h_in.p, bytes, cudaMemcpyHostToDevice, s),
            "H2D offsets");
    PF_CUDA(cudaEventRecord(ctx->ev_staged, s), "event");
    ctx->staged_pending = true;
    *d_off = (const int64_t*)ctx->d_in.p;
    *max_len = (uint32_t)mx;
    return PF_OK;
}

int ls_common_checks(pf_ctx* ctx, const float* d_times, const int64_t* offsets,
                     uint64_t n_curves, const void* d_omega, uint64_t n_freq) {
    if (!ctx) return PF_EINVAL;
    if (n_curves == 0 || n_freq == 0) return PF_OK;
    if (!offsets) return fail(ctx, PF_EINVAL, "offsets is NULL");
    if (!d_omega) return fail(ctx, PF_EINVAL, "omega is NULL");
    if (offsets[n_curves] > offsets[0] && !d_times) return fail(ctx, PF_EINVAL, "d_times is NULL");
    return PF_OK;
}

// FPW for host-pointer inputs (FPW::CalcFPWBatched, periodfind/cuda/fpw.cu;
// calc_fpw_batched / calc_fpw_peaks_batched, rust/src/lib.rs:202-256,
// 680-720).  The host computes the per-point weights as both references do
// (iv = 1 / err^2, ivy = iv * m, errs absent = 1), packs them with the
// times, and one launch covers every (curve, period derivative, period
// tile); the peaks, when asked for, are found on the device.
//
// BLS (BLS::CalcBLSBatched, periodfind/cuda/bls.cu; calc_bls_batched /
// calc_bls_peaks_batched, rust/src/lib.rs:264-322, 718-760) runs the same
// way with the second weight w * (m - mean), mean = sum(w m) / sum(w) in
// sequential f32 sums as both references compute it (bls.rs:36-48,
// bls.cu:419-435), and the window search of the kernel.
int run_fpw(pf_ctx* ctx, const float* const* times, const float* const* mags,
            const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
            const float* periods, uint64_t n_per, const float* pdts, uint64_t n_pdt,
            uint32_t n_bins, int mode, float* out, bool peaks, uint32_t n_peaks,
            uint32_t min_distance, int64_t* out_idx, float* out_val, bool bls = false,
            float qmin = 0.0f, float qmax = 0.0f) {
    if (!ctx) return PF_EINVAL;
    ctx->res_copies.clear();
    Job j;
    j.algo = ALGO_LS;  // no bin-count checks of CE / AOV apply
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = periods;
    j.n_per = n_per;
    j.pdts = pdts;
    j.n_pdt = n_pdt;
    j.peaks = peaks;
    j.n_peaks = n_peaks;
    j.out_idx = out_idx;
    j.out_val = out_val;
    j.out = out;
    int rc = validate_common(ctx, j);
    if (rc != PF_OK) return rc;
    if (mode & PF_TIMING) return fail(ctx, PF_EINVAL, "PF_TIMING does not apply to FPW / BLS");
    const bool async = (mode & PF_ASYNC) != 0;
    if (async) {
        if (!peaks) return fail(ctx, PF_EINVAL, "PF_ASYNC applies to the peak calls only");
        if (ctx->pend_count == pf_ctx::kMaxPending)
            return fail(ctx, PF_EINVAL, "%d PF_ASYNC calls are pending; collect one with pf_wait",
                        pf_ctx::kMaxPending);
    }
    if (n_bins < 1 || n_bins > kFpwMaxBins)
        return fail(ctx, PF_EINVAL, "n_bins must be in [1, %u], got %u", kFpwMaxBins, n_bins);
    if (n_curves == 0) return async ? push_pending(ctx, j, 0, false, nullptr) : PF_OK;
    if (!times || !mags || !lengths) return fail(ctx, PF_EINVAL, "times/mags/lengths is NULL");
    const uint64_t n_cells = n_per * n_pdt;
    if (n_cells == 0) return async ? push_pending(ctx, j, 0, false, nullptr) : PF_OK;
    if ((rc = check_grid_host(ctx, j)) != PF_OK) return rc;
    std::vector<int64_t> off(n_curves);
    std::vector<uint32_t> len(n_curves);
    uint64_t total = 0;
    for (uint64_t c = 0; c < n_curves; c++) {
        if (lengths[c] > 0xFFFFFFFFull)
            return fail(ctx, PF_EINVAL, "a curve has more than 2^32-1 points");
        if (lengths[c] > 0 && (!times[c] || !mags[c]))
            return fail(ctx, PF_EINVAL, "curve %llu has a NULL array", (unsigned long long)c);
        off[c] = (int64_t)total;
        len[c] = (uint32_t)lengths[c];
        total += lengths[c];
    }
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const size_t o_iv = align_up(total * 4, 256), o_ivy = o_iv + align_up(total * 4, 256);
    const size_t o_off = o_ivy + align_up(total * 4, 256);
    const size_t o_len = o_off + align_up(n_curves * 8, 256);
    const size_t o_per = o_len + align_up(n_curves * 4, 256);
    const size_t o_pdt = o_per + align_up(n_per * 4, 256);
    const size_t bytes = o_pdt + align_up(n_pdt * 4, 256);
    if ((rc = staging_ready(ctx)) != PF_OK) return rc;
    if ((rc = ensure_pinned(ctx, ctx->h_in, bytes)) != PF_OK) return rc;
    const int slot = ctx->in_slot;  // the input block (see run_host)
    DevBuf& din = slot ? ctx->d_in2 : ctx->d_in;
    if ((rc = ensure_dev(ctx, din, bytes)) != PF_OK) return rc;
    char* hb = (char*)ctx->h_in.p;
    float* ht = (float*)hb;
    float* hiv = (float*)(hb + o_iv);
    float* hivy = (float*)(hb + o_ivy);
    double tmax = 0.0;
    {
        const CurveTasks T = curve_tasks(off, total);
        std::vector<int> bad(T.count(), 0);
        std::vector<float> tmx(T.count(), 0.0f);
        auto worker = [&](unsigned w) {
            for (uint64_t c = T.first[w]; c < T.first[w + 1]; c++) {
                const float* t = times[c];
                const float* m = mags[c];
                const float* e = errs ? errs[c] : nullptr;
                const int64_t o = off[c];
                // This unit is built without multiply-add contraction.
                float mean_y = 0.0f;
                if (bls) {
                    float total_w = 0.0f, total_wy = 0.0f;
                    for (uint32_t i = 0; i < len[c]; i++) {
                        const float err = e ? e[i] : 1.0f;
                        const float w_i = 1.0f / (err * err);
                        total_w += w_i;
                        total_wy += w_i * m[i];
                    }
                    mean_y = total_w > 0.0f ? total_wy / total_w : 0.0f;
                }
                for (uint32_t i = 0; i < len[c]; i++) {
                    const float x = t[i];
                    if (!std::isfinite(x)) bad[w] = 1;
                    tmx[w] = std::max(tmx[w], std::fabs(x));
                    ht[o + i] = x;
                    const float err = e ? e[i] : 1.0f;
                    const float w_i = 1.0f / (err * err);
                    hiv[o + i] = w_i;
                    hivy[o + i] = bls ? w_i * (m[i] - mean_y) : w_i * m[i];
                }
            }
        };
        ctx->pool.run(T.count(), T.width, worker);
        for (int b : bad)
            if (b) return fail(ctx, PF_EINVAL, "times must be finite");
        for (float x : tmx) tmax = std::max(tmax, (double)x);
    }
    memcpy(hb + o_off, off.data(), n_curves * 8);
    memcpy(hb + o_len, len.data(), n_curves * 4);
    memcpy(hb + o_per, periods, n_per * 4);
    memcpy(hb + o_pdt, pdts, n_pdt * 4);
    cudaStream_t s = ctx->stream;
    char* db = (char*)din.p;
    if ((rc = order_after_previous(ctx, s)) != PF_OK) return rc;
    // As run_host: the copy on the copy stream after this block's last
    // reader, the kernels after the copy.
    CallEnd call_end{ctx, s};
    PF_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev_in_free[slot], 0), "stream wait");
    PF_CUDA(cudaMemcpyAsync(db, hb, bytes, cudaMemcpyHostToDevice, ctx->copy_stream),
            "H2D inputs");
    PF_CUDA(cudaEventRecord(ctx->ev_copied[slot], ctx->copy_stream), "event");
    PF_CUDA(cudaEventRecord(ctx->ev_staged, ctx->copy_stream), "event");
    ctx->staged_pending = true;
    ctx->in_slot = slot ^ 1;
    PF_CUDA(cudaStreamWaitEvent(s, ctx->ev_copied[slot], 0), "stream wait");
    const size_t out_bytes = (size_t)n_curves * n_cells * 4;
    if ((rc = ensure_dev(ctx, ctx->d_out, out_bytes)) != PF_OK) return rc;
    FpwParams p{};
    p.t = (const float*)db;
    p.iv = (const float*)(db + o_iv);
    p.ivy = (const float*)(db + o_ivy);
    p.off = (const int64_t*)(db + o_off);
    p.len = (const uint32_t*)(db + o_len);
    p.periods = (const float*)(db + o_per);
    p.pdts = (const float*)(db + o_pdt);
    p.n_per = n_per;
    p.n_pdt = (uint32_t)n_pdt;
    p.n_bins = n_bins;
    // FPW::FPW (fpw.cu:19-22): 1.0 / (float)n_bins in double, stored as
    // float; BLS::BLS (bls.cu:20-25): 1.0f / (float)n_bins.
    p.bin_size = bls ? 1.0f / (float)n_bins : (float)(1.0 / (double)(float)n_bins);
    p.bls = bls ? 1 : 0;
    if (bls) {
        // Window widths (bls.rs:51-52): max(floor(qmin nb), 1) and
        // min(ceil(qmax nb), nb - 1), with Rust's saturating float casts.
        auto sat = [](float x) -> uint64_t {
            if (!(x > 0.0f)) return 0;
            if (x >= 18446744073709551616.0f) return UINT64_MAX;
            return (uint64_t)x;
        };
        p.nb_min = (uint32_t)std::max<uint64_t>(sat(std::floor(qmin * (float)n_bins)), 1);
        p.nb_max = (uint32_t)std::min<uint64_t>(sat(std::ceil(qmax * (float)n_bins)), n_bins - 1);
    }
    p.out = (float*)ctx->d_out.p;
    p.tmax = tmax;
    p.edge_d = edge_guard(n_bins);
    const bool exact = (mode & PF_MODE_CHOSEN) != 0;
    PF_CUDA(cudaEventRecord(ctx->ev0, s), "event");
    PF_CUDA((mode & PF_SEM_CPU) ? launch_fpw_cpusem(p, exact, n_curves, s)
                                : launch_fpw_cudasem(p, exact, n_curves, s),
            "FPW / BLS kernel launch");
    PF_CUDA(cudaEventRecord(ctx->ev1, s), "event");
    ctx->timed_pending = true;
    ctx->launches++;
    if (peaks) {
        if (n_peaks > 0) {
            const size_t pk = (size_t)n_curves * n_peaks;
            if ((rc = ensure_dev(ctx, ctx->d_pidx, pk * 8)) != PF_OK) return rc;
            if ((rc = ensure_dev(ctx, ctx->d_pval, pk * 4)) != PF_OK) return rc;
            PF_CUDA(launch_peaks(p.out, n_curves, n_cells, n_peaks, min_distance, 1,
                                 (int64_t*)ctx->d_pidx.p, (float*)ctx->d_pval.p, s),
                    "peak search launch");
            ctx->launches++;
        }
        if ((rc = copy_peaks_back(ctx, j, async, s)) != PF_OK) return rc;
        if (async) {
            ctx->cur_slot = slot;
            call_end.armed = false;
            return mark_done(ctx, s);
        }
    } else {
        PF_CUDA(cudaMemcpyAsync(out, p.out, out_bytes, cudaMemcpyDeviceToHost, s),
                "D2H periodogram");
    }
    ctx->cur_slot = slot;
    call_end.armed = false;
    return finish_sync(ctx, s);
}

}  // namespace

size_t pfk::fold_smem(const FoldConfig& c, uint32_t n_phase, uint32_t n_mag) {
    if (c.kind == KIND_LSREC) return kRecTileBytes;
    if (c.kind == KIND_BINWARP)
        return (size_t)kWarpMaxPoints * 16 +
               (size_t)(c.block / 32) * (c.algo == ALGO_CE ? n_phase * n_mag : 2 * n_phase) * 4;
    if (c.kind == KIND_BIN) return bin_smem_bytes(c.algo, c.cnt16, c.block, n_phase, n_mag);
    return fold_smem_bytes(c.algo, c.fold, c.acc, c.block, c.ovl, n_phase, n_mag);
}

// ------------------------------------------------------------------ C ABI

extern "C" {

int pf_version(void) { return 100; }

int pf_ctx_create(pf_ctx** out, int device) {
    if (!out) return PF_EINVAL;
    *out = nullptr;
    int n_dev = 0;
    cudaError_t e = cudaGetDeviceCount(&n_dev);
    if (e != cudaSuccess || n_dev == 0) {
        cudaGetLastError();
        g_create_error = std::string("no CUDA device available: ") + cudaGetErrorString(e);
        return PF_ECUDA;
    }
    if (device < 0 || device >= n_dev) {
        g_create_error = "device index out of range";
        return PF_EINVAL;
    }
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) {
        g_create_error = cudaGetErrorString(e);
        return PF_ECUDA;
    }
    if (prop.major != 10) {
        g_create_error = "this library is built for sm_100a (B200); device is sm_" +
                         std::to_string(prop.major) + std::to_string(prop.minor);
        return PF_EUNSUPPORTED;
    }
    pf_ctx* ctx = new pf_ctx();
    ctx->device = device;
    ctx->n_sm = prop.multiProcessorCount;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    if ((e = cudaSetDevice(device)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&ctx->ev0)) != cudaSuccess ||
        (e = cudaEventCreate(&ctx->ev1)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_staged, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_done, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->pend[0].done, cudaEventDisableTiming)) !=
            cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->pend[1].done, cudaEventDisableTiming)) !=
            cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_prep, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_in_free[0], cudaEventDisableTiming)) !=
            cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_in_free[1], cudaEventDisableTiming)) !=
            cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_copied[0], cudaEventDisableTiming)) !=
            cudaSuccess ||
        (e = cudaEventCreateWithFlags(&ctx->ev_copied[1], cudaEventDisableTiming)) !=
            cudaSuccess) {
        g_create_error = cudaGetErrorString(e);
        pf_ctx_destroy(ctx);
        return PF_ECUDA;
    }
    *out = ctx;
    return PF_OK;
}

void pf_ctx_destroy(pf_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    if (ctx->done_recorded) cudaEventSynchronize(ctx->ev_done);
    if (ctx->prep_pending) cudaEventSynchronize(ctx->ev_prep);
    for (DevBuf* b : {&ctx->d_in, &ctx->d_aux32, &ctx->d_aux64, &ctx->d_out, &ctx->d_pidx,
                      &ctx->d_pval, &ctx->d_pack, &ctx->d_misc, &ctx->d_stamps, &ctx->d_stat, &ctx->d_bins,
                      &ctx->d_prep, &ctx->d_in2})
        if (b->p) cudaFree(b->p);
    if (ctx->h_in.p) cudaFreeHost(ctx->h_in.p);
    if (ctx->h_res.p) cudaFreeHost(ctx->h_res.p);
    for (pf_ctx::Pending& q : ctx->pend) {
        if (q.res.p) cudaFreeHost(q.res.p);
        if (q.done) cudaEventDestroy(q.done);
    }
    if (ctx->ev_prep) cudaEventDestroy(ctx->ev_prep);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->ev_staged) cudaEventDestroy(ctx->ev_staged);
    if (ctx->ev_done) cudaEventDestroy(ctx->ev_done);
    for (cudaEvent_t ev : {ctx->ev_in_free[0], ctx->ev_in_free[1], ctx->ev_copied[0],
                           ctx->ev_copied[1]})
        if (ev) cudaEventDestroy(ev);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* pf_last_error(const pf_ctx* ctx) {
    if (!ctx) return g_create_error.c_str();
    return ctx->err.c_str();
}

uint64_t pf_launch_count(const pf_ctx* ctx) { return ctx ? ctx->launches : 0; }

int pf_normalize_mags(const float* const* mags, const uint64_t* lengths, uint64_t n_curves,
                      float* const* out) {
    if (n_curves == 0) return PF_OK;
    if (!mags || !lengths || !out) return PF_EINVAL;
    uint64_t total = 0;
    for (uint64_t c = 0; c < n_curves; c++) {
        if (lengths[c] == 0) return PF_EINVAL;  // numpy's min/max of an empty array raise
        if (!mags[c] || !out[c]) return PF_EINVAL;
        total += lengths[c];
    }
    auto one = [&](uint64_t c) { normalize_curve(mags[c], lengths[c], out[c]); };
    for_each_curve(n_curves, total, one);
    return PF_OK;
}

int pf_center_mags(const float* const* mags, const uint64_t* lengths, uint64_t n_curves,
                   float* const* out) {
    if (n_curves == 0) return PF_OK;
    if (!mags || !lengths || !out) return PF_EINVAL;
    uint64_t total = 0;
    for (uint64_t c = 0; c < n_curves; c++) {
        if (lengths[c] == 0 || !mags[c] || !out[c]) return PF_EINVAL;
        total += lengths[c];
    }
    auto one = [&](uint64_t c) { center_curve(mags[c], lengths[c], out[c]); };
    for_each_curve(n_curves, total, one);
    return PF_OK;
}

int pf_tuning_report(const pf_ctx* ctx, char* buf, uint64_t len) {
    if (!ctx) return PF_EINVAL;
    std::string out;
    for (const auto& kv : ctx->tuned) {
        char line[320];
        snprintf(line, sizeof(line),
                 "%s: %sblock=%d rounds=%d %s sample_ms=%.3f slowest_ms=%.3f candidates=%u\n",
                 kv.first.c_str(),
                 kv.second.kind == KIND_LSREC ? "trig=recurrence "
                 : kv.second.kind == KIND_BINWARP ? "bins=shared-atomic "
                 : kv.second.kind == KIND_BIN ? "bins=privatised "
                 : (kv.second.kind == KIND_FOLD && kv.first.find("fgrid") != std::string::npos)
                     ? "trig=sincos "
                     : "",
                 kv.second.block, kv.second.rounds,
                 kv.second.persist ? "persistent" : "one-cta-per-item", kv.second.ms,
                 kv.second.ms_worst, kv.second.candidates);
        out += line;
    }
    if (buf && len > 0) {
        const size_t n = std::min<size_t>(out.size(), (size_t)len - 1);
        memcpy(buf, out.data(), n);
        buf[n] = '\0';
    }
    return (int)ctx->tuned.size();
}

int pf_curve_latency(pf_ctx* ctx, uint64_t n_curves, double* out_ns) {
    if (!ctx || (!out_ns && n_curves)) return PF_EINVAL;
    const size_t nw = ctx->stamp_curves.size();
    if (nw == 0) return fail(ctx, PF_EINVAL, "no launch with PF_TIMING on this context");
    if (n_curves != ctx->stamp_n_curves)
        return fail(ctx, PF_EINVAL, "n_curves differs from the last PF_TIMING launch");
    std::vector<unsigned long long> st(2 * nw);
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    PF_CUDA(cudaMemcpyAsync(st.data(), ctx->d_stamps.p, nw * 16, cudaMemcpyDeviceToHost,
                            ctx->stamp_stream),
            "D2H stamps");
    PF_CUDA(cudaStreamSynchronize(ctx->stamp_stream), "stream synchronize");
    std::vector<unsigned long long> lo(n_curves, ~0ull), hi(n_curves, 0ull);
    for (size_t k = 0; k < nw; k++) {
        const uint32_t c = ctx->stamp_curves[k];
        if (c >= n_curves) continue;
        lo[c] = std::min(lo[c], st[2 * k]);
        hi[c] = std::max(hi[c], st[2 * k + 1]);
    }
    for (uint64_t c = 0; c < n_curves; c++)
        out_ns[c] = (hi[c] > lo[c] && lo[c] != ~0ull) ? (double)(hi[c] - lo[c]) : 0.0;
    return PF_OK;
}

int pf_ls_eval_dev(pf_ctx* ctx, const float* d_times, const float* d_mags,
                   const int64_t* offsets, uint64_t n_curves, const double* d_omega,
                   uint64_t omega_stride, uint64_t n_freq, float* d_power, float* d_dpdw,
                   float* d_d2pdw2, float* d_coef, void* stream) {
    int rc = ls_common_checks(ctx, d_times, offsets, n_curves, d_omega, n_freq);
    if (rc != PF_OK || n_curves == 0 || n_freq == 0) return rc;
    if (!d_power) return fail(ctx, PF_EINVAL, "d_power is NULL");
    if (offsets[n_curves] > offsets[0] && !d_mags) return fail(ctx, PF_EINVAL, "d_mags is NULL");
    if (omega_stride != 0 && omega_stride < n_freq)
        return fail(ctx, PF_EINVAL, "omega_stride must be 0 or >= n_freq");
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    LsEvalParams p;
    uint32_t max_len = 0;
    if ((rc = stage_offsets(ctx, offsets, n_curves, s, &p.off, &max_len)) != PF_OK) return rc;
    p.t = d_times;
    p.y = d_mags;
    p.n_curves = n_curves;
    p.omega = d_omega;
    p.omega_stride = omega_stride;
    p.n_freq = n_freq;
    p.power = d_power;
    p.dpdw = d_dpdw;
    p.d2pdw2 = d_d2pdw2;
    p.coef = d_coef;
    const int order = d_d2pdw2 ? 2 : (d_dpdw ? 1 : 0);
    PF_CUDA(launch_ls_eval(p, order, s), "LS derivative kernel");
    ctx->launches++;
    return mark_done(ctx, s);
}

int pf_ls_backward_dev(pf_ctx* ctx, const float* d_times, const int64_t* offsets,
                       uint64_t n_curves, const double* d_omega, uint64_t omega_stride,
                       uint64_t n_freq, const float* d_grad_power, const float* d_dpdw,
                       const float* d_coef, double* d_grad_omega, float* d_grad_mags,
                       void* stream) {
    int rc = ls_common_checks(ctx, d_times, offsets, n_curves, d_omega, n_freq);
    if (rc != PF_OK || n_curves == 0 || n_freq == 0) return rc;
    if (!d_grad_power || !d_coef) return fail(ctx, PF_EINVAL, "d_grad_power/d_coef is NULL");
    if (d_grad_omega && !d_dpdw) return fail(ctx, PF_EINVAL, "d_grad_omega needs d_dpdw");
    if (omega_stride != 0 && omega_stride < n_freq)
        return fail(ctx, PF_EINVAL, "omega_stride must be 0 or >= n_freq");
    if (!d_grad_omega && !d_grad_mags) return PF_OK;
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    LsGradParams p;
    uint32_t max_len = 0;
    if ((rc = stage_offsets(ctx, offsets, n_curves, s, &p.off, &max_len)) != PF_OK) return rc;
    p.t = d_times;
    p.n_curves = n_curves;
    p.omega = d_omega;
    p.omega_stride = omega_stride;
    p.n_freq = n_freq;
    p.grad_power = d_grad_power;
    p.dpdw = d_dpdw;
    p.coef = d_coef;
    p.grad_omega = d_grad_omega;
    p.grad_mags = d_grad_mags;
    PF_CUDA(launch_ls_grad(p, max_len, s), "LS backward kernel");
    ctx->launches++;
    return mark_done(ctx, s);
}

int pf_ls_refine_dev(pf_ctx* ctx, const float* d_times, const float* d_mags,
                     const int64_t* offsets, uint64_t n_curves, const double* d_omega0,
                     const double* d_half_width, uint64_t n_freq, uint32_t n_steps,
                     double* d_omega, float* d_power, void* stream) {
    int rc = ls_common_checks(ctx, d_times, offsets, n_curves, d_omega0, n_freq);
    if (rc != PF_OK || n_curves == 0 || n_freq == 0) return rc;
    if (!d_half_width || !d_omega || !d_power)
        return fail(ctx, PF_EINVAL, "d_half_width/d_omega/d_power is NULL");
    if (offsets[n_curves] > offsets[0] && !d_mags) return fail(ctx, PF_EINVAL, "d_mags is NULL");
    if (n_steps > 64) return fail(ctx, PF_EINVAL, "n_steps must be <= 64");
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    LsEvalParams p;
    uint32_t max_len = 0;
    if ((rc = stage_offsets(ctx, offsets, n_curves, s, &p.off, &max_len)) != PF_OK) return rc;
    p.t = d_times;
    p.y = d_mags;
    p.n_curves = n_curves;
    p.omega = d_omega0;
    p.omega_stride = n_freq;
    p.n_freq = n_freq;
    p.power = d_power;
    p.half_width = d_half_width;
    p.n_steps = n_steps;
    p.omega_out = d_omega;
    PF_CUDA(launch_ls_refine(p, s), "LS Newton refinement kernel");
    ctx->launches++;
    return mark_done(ctx, s);
}

int pf_fold_phase_dev(pf_ctx* ctx, int mode, const float* d_times, uint64_t n,
                      const float* d_periods, uint64_t n_per, float period_dt, float* d_out,
                      void* stream) {
    if (!ctx) return PF_EINVAL;
    if (n == 0 || n_per == 0) return PF_OK;
    if (!d_times || !d_periods || !d_out) return fail(ctx, PF_EINVAL, "NULL pointer argument");
    const int f = mode & (PF_FOLD_F32 | PF_FOLD_DF | PF_FOLD_EXACT);
    int fold;
    if (f == 0) fold = FOLD_REF;
    else if (f == PF_FOLD_F32) fold = FOLD_F32;
    else if (f == PF_FOLD_DF) fold = FOLD_DF;
    else if (f == PF_FOLD_EXACT) fold = FOLD_EXACT;
    else return fail(ctx, PF_EINVAL, "at most one of PF_FOLD_F32 / PF_FOLD_DF / PF_FOLD_EXACT");
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    PF_CUDA(use_cpu_semantics(mode)
                ? launch_phase_probe_cpusem(fold, d_times, n, d_periods, n_per, period_dt, d_out, s)
                : launch_phase_probe_cudasem(fold, d_times, n, d_periods, n_per, period_dt, d_out,
                                             s),
            "phase probe kernel");
    ctx->launches++;
    return PF_OK;
}

double pf_last_kernel_ms(const pf_ctx* ctx) {
    if (!ctx) return -1.0;
    pf_ctx* c = const_cast<pf_ctx*>(ctx);
    if (c->timed_pending && cudaEventQuery(c->ev1) == cudaSuccess) read_kernel_time(c);
    return c->last_ms;
}

int pf_ce(pf_ctx* ctx, const float* const* times, const float* const* mags,
          const uint64_t* lengths, uint64_t n_curves, const float* periods, uint64_t n_per,
          const float* period_dts, uint64_t n_pdt, uint32_t n_phase, uint32_t n_mag,
          uint32_t phase_overlap, uint32_t mag_overlap, int mode, float* out) {
    Job j;
    j.algo = ALGO_CE;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = periods;
    j.n_per = n_per;
    j.pdts = period_dts;
    j.n_pdt = n_pdt;
    j.n_phase = n_phase;
    j.n_mag = n_mag;
    j.po = phase_overlap;
    j.mo = mag_overlap;
    j.out = out;
    return run_host(ctx, j, times, mags, lengths);
}

int pf_aov(pf_ctx* ctx, const float* const* times, const float* const* mags,
           const uint64_t* lengths, uint64_t n_curves, const float* periods, uint64_t n_per,
           const float* period_dts, uint64_t n_pdt, uint32_t n_phase, uint32_t phase_overlap,
           int mode, float* out) {
    Job j;
    j.algo = ALGO_AOV;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = periods;
    j.n_per = n_per;
    j.pdts = period_dts;
    j.n_pdt = n_pdt;
    j.n_phase = n_phase;
    j.po = phase_overlap;
    j.out = out;
    return run_host(ctx, j, times, mags, lengths);
}

int pf_ls_fgrid(pf_ctx* ctx, const float* const* times, const float* const* mags,
                const uint64_t* lengths, uint64_t n_curves, double f_min, double df,
                uint64_t n_freq, int mode, float* out) {
    static const float kZeroPdt = 0.0f;
    Job j;
    j.algo = ALGO_LS;
    j.mode = mode;
    j.n_curves = n_curves;
    j.n_per = n_freq;
    j.pdts = &kZeroPdt;
    j.n_pdt = 1;
    j.fgrid = true;
    j.f0 = f_min;
    j.df = df;
    j.out = out;
    return run_host(ctx, j, times, mags, lengths);
}

int pf_ls_fgrid_dev(pf_ctx* ctx, const float* d_times, const float* d_mags,
                    const int64_t* offsets, uint64_t n_curves, double f_min, double df,
                    uint64_t n_freq, int mode, float* d_out, void* stream) {
    Job j;
    j.algo = ALGO_LS;
    j.mode = mode;
    j.n_curves = n_curves;
    j.n_per = n_freq;
    j.n_pdt = 1;
    j.fgrid = true;
    j.f0 = f_min;
    j.df = df;
    j.out = d_out;
    return run_dev(ctx, j, d_times, d_mags, offsets, stream);
}

int pf_bin_counts(pf_ctx* ctx, int algo, const float* const* times, const float* const* mags,
                  const uint64_t* lengths, uint64_t n_curves, const float* periods,
                  uint64_t n_per, const float* period_dts, uint64_t n_pdt, uint32_t n_phase,
                  uint32_t n_mag, uint32_t phase_overlap, uint32_t mag_overlap, int mode,
                  float* out, uint32_t* out_counts) {
    if (!ctx) return PF_EINVAL;
    if (algo != PF_ALGO_CE && algo != PF_ALGO_AOV)
        return fail(ctx, PF_EINVAL, "bin counts exist for PF_ALGO_CE and PF_ALGO_AOV only");
    if (mode & (PF_ASYNC | PF_TIMING))
        return fail(ctx, PF_EINVAL, "PF_ASYNC / PF_TIMING do not apply to pf_bin_counts");
    if (n_curves > 0 && n_per > 0 && n_pdt > 0 && !out_counts)
        return fail(ctx, PF_EINVAL, "out_counts is NULL");
    Job j;
    j.algo = algo == PF_ALGO_CE ? ALGO_CE : ALGO_AOV;
    // The chosen form writes its counts from the reference-statistic epilogue.
    j.mode = (mode & PF_MODE_CHOSEN) ? (mode | PF_REF_STATS) : mode;
    j.n_curves = n_curves;
    j.periods = periods;
    j.n_per = n_per;
    j.pdts = period_dts;
    j.n_pdt = n_pdt;
    j.n_phase = n_phase;
    j.n_mag = algo == PF_ALGO_CE ? n_mag : 1;
    j.po = phase_overlap;
    j.mo = algo == PF_ALGO_CE ? mag_overlap : 1;
    j.out = out;
    j.out_bins = out_counts;
    return run_host(ctx, j, times, mags, lengths);
}

int pf_ls(pf_ctx* ctx, const float* const* times, const float* const* mags,
          const uint64_t* lengths, uint64_t n_curves, const float* periods, uint64_t n_per,
          const float* period_dts, uint64_t n_pdt, int mode, float* out) {
    Job j;
    j.algo = ALGO_LS;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = periods;
    j.n_per = n_per;
    j.pdts = period_dts;
    j.n_pdt = n_pdt;
    j.out = out;
    return run_host(ctx, j, times, mags, lengths);
}

int pf_ce_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                const uint64_t* lengths, uint64_t n_curves, const float* periods,
                uint64_t n_per, const float* period_dts, uint64_t n_pdt, uint32_t n_phase,
                uint32_t n_mag, uint32_t phase_overlap, uint32_t mag_overlap, uint32_t n_peaks,
                uint32_t min_distance, int mode, int64_t* out_idx, float* out_val) {
    Job j;
    j.algo = ALGO_CE;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = periods;
    j.n_per = n_per;
    j.pdts = period_dts;
    j.n_pdt = n_pdt;
    j.n_phase = n_phase;
    j.n_mag = n_mag;
    j.po = phase_overlap;
    j.mo = mag_overlap;
    j.peaks = true;
    j.n_peaks = n_peaks;
    j.min_distance = min_distance;
    j.out_idx = out_idx;
    j.out_val = out_val;
    return run_host(ctx, j, times, mags, lengths);
}

int pf_aov_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                 const uint64_t* lengths, uint64_t n_curves, const float* periods,
                 uint64_t n_per, const float* period_dts, uint64_t n_pdt, uint32_t n_phase,
                 uint32_t phase_overlap, uint32_t n_peaks, uint32_t min_distance, int mode,
                 int64_t* out_idx, float* out_val) {
    Job j;
    j.algo = ALGO_AOV;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = periods;
    j.n_per = n_per;
    j.pdts = period_dts;
    j.n_pdt = n_pdt;
    j.n_phase = n_phase;
    j.po = phase_overlap;
    j.peaks = true;
    j.n_peaks = n_peaks;
    j.min_distance = min_distance;
    j.out_idx = out_idx;
    j.out_val = out_val;
    return run_host(ctx, j, times, mags, lengths);
}

int pf_ls_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                const uint64_t* lengths, uint64_t n_curves, const float* periods,
                uint64_t n_per, const float* period_dts, uint64_t n_pdt, uint32_t n_peaks,
                uint32_t min_distance, int mode, int64_t* out_idx, float* out_val) {
    Job j;
    j.algo = ALGO_LS;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = periods;
    j.n_per = n_per;
    j.pdts = period_dts;
    j.n_pdt = n_pdt;
    j.peaks = true;
    j.n_peaks = n_peaks;
    j.min_distance = min_distance;
    j.out_idx = out_idx;
    j.out_val = out_val;
    return run_host(ctx, j, times, mags, lengths);
}

int pf_fpw(pf_ctx* ctx, const float* const* times, const float* const* mags,
           const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
           const float* periods, uint64_t n_per, const float* period_dts, uint64_t n_pdt,
           uint32_t n_bins, int mode, float* out) {
    return run_fpw(ctx, times, mags, errs, lengths, n_curves, periods, n_per, period_dts, n_pdt,
                   n_bins, mode, out, false, 0, 0, nullptr, nullptr);
}

int pf_fpw_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                 const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
                 const float* periods, uint64_t n_per, const float* period_dts, uint64_t n_pdt,
                 uint32_t n_bins, uint32_t n_peaks, uint32_t min_distance, int mode,
                 int64_t* out_idx, float* out_val) {
    return run_fpw(ctx, times, mags, errs, lengths, n_curves, periods, n_per, period_dts, n_pdt,
                   n_bins, mode, nullptr, true, n_peaks, min_distance, out_idx, out_val);
}

int pf_prepare_mags_dev(pf_ctx* ctx, const float* d_mags, const int64_t* offsets,
                        uint64_t n_curves, int kind, float* d_out, void* stream) {
    if (!ctx) return PF_EINVAL;
    if (kind != PF_PREP_CENTER && kind != PF_PREP_NORMALIZE)
        return fail(ctx, PF_EINVAL, "kind must be PF_PREP_CENTER or PF_PREP_NORMALIZE");
    if (n_curves == 0) return PF_OK;
    if (!offsets) return fail(ctx, PF_EINVAL, "offsets is NULL");
    if (n_curves > 0x7FFFFFFFull) return fail(ctx, PF_EINVAL, "too many curves");
    if (offsets[0] < 0) return fail(ctx, PF_EINVAL, "offsets[0] is negative");
    uint32_t leaf_cap = 1;
    for (uint64_t c = 0; c < n_curves; c++) {
        const int64_t len = offsets[c + 1] - offsets[c];
        if (len < 0 || len > 0xFFFFFFFFll)
            return fail(ctx, PF_EINVAL, "offsets must be non-decreasing (curve %llu)",
                        (unsigned long long)c);
        if (kind == PF_PREP_CENTER && len > 0)
            leaf_cap = std::max(leaf_cap, stats_leaf_count((uint32_t)len));
    }
    if ((size_t)leaf_cap * 12 > 200u * 1024u)
        return fail(ctx, PF_EUNSUPPORTED, "a curve is too long for the device mean");
    if (offsets[n_curves] > offsets[0] && (!d_mags || !d_out))
        return fail(ctx, PF_EINVAL, "d_mags / d_out is NULL");
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (ctx->prep_pending) {
        PF_CUDA(cudaEventSynchronize(ctx->ev_prep), "previous preparation");
        ctx->prep_pending = false;
    }
    int rc;
    if ((rc = ensure_dev(ctx, ctx->d_prep, (n_curves + 1) * 8)) != PF_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    PF_CUDA(cudaMemcpyAsync(ctx->d_prep.p, offsets, (n_curves + 1) * 8, cudaMemcpyHostToDevice,
                            s),
            "H2D offsets");
    PF_CUDA(launch_prep_mags(d_mags, (const int64_t*)ctx->d_prep.p, n_curves, leaf_cap, kind,
                             d_out, s),
            "magnitude preparation launch");
    PF_CUDA(cudaEventRecord(ctx->ev_prep, s), "event");
    ctx->prep_pending = true;
    ctx->launches++;
    return PF_OK;
}

int pf_bls(pf_ctx* ctx, const float* const* times, const float* const* mags,
           const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
           const float* periods, uint64_t n_per, const float* period_dts, uint64_t n_pdt,
           uint32_t n_bins, float qmin, float qmax, int mode, float* out) {
    return run_fpw(ctx, times, mags, errs, lengths, n_curves, periods, n_per, period_dts, n_pdt,
                   n_bins, mode, out, false, 0, 0, nullptr, nullptr, true, qmin, qmax);
}

int pf_bls_peaks(pf_ctx* ctx, const float* const* times, const float* const* mags,
                 const float* const* errs, const uint64_t* lengths, uint64_t n_curves,
                 const float* periods, uint64_t n_per, const float* period_dts, uint64_t n_pdt,
                 uint32_t n_bins, float qmin, float qmax, uint32_t n_peaks,
                 uint32_t min_distance, int mode, int64_t* out_idx, float* out_val) {
    return run_fpw(ctx, times, mags, errs, lengths, n_curves, periods, n_per, period_dts, n_pdt,
                   n_bins, mode, nullptr, true, n_peaks, min_distance, out_idx, out_val, true,
                   qmin, qmax);
}

int pf_wait(pf_ctx* ctx) {
    if (!ctx) return PF_EINVAL;
    if (ctx->pend_count == 0) return fail(ctx, PF_EINVAL, "no PF_ASYNC call is pending");
    pf_ctx::Pending& q = ctx->pend[ctx->pend_head];
    ctx->pend_head = (ctx->pend_head + 1) % pf_ctx::kMaxPending;
    ctx->pend_count--;
    if (!q.work) return PF_OK;
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    PF_CUDA(cudaEventSynchronize(q.done), "asynchronous peak call");
    if (q.n > 0) {
        const char* hr = (const char*)q.res.p;
        memcpy(q.out_idx, hr, q.n * 8);
        memcpy(q.out_val, hr + q.n * 8, q.n * 4);
    }
    return PF_OK;
}

int pf_ce_dev(pf_ctx* ctx, const float* d_times, const float* d_mags, const int64_t* offsets,
              uint64_t n_curves, const float* d_periods, uint64_t n_per, const float* d_pdts,
              uint64_t n_pdt, uint32_t n_phase, uint32_t n_mag, uint32_t phase_overlap,
              uint32_t mag_overlap, int mode, float* d_out, void* stream) {
    Job j;
    j.algo = ALGO_CE;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = d_periods;
    j.n_per = n_per;
    j.pdts = d_pdts;
    j.n_pdt = n_pdt;
    j.n_phase = n_phase;
    j.n_mag = n_mag;
    j.po = phase_overlap;
    j.mo = mag_overlap;
    j.out = d_out;
    return run_dev(ctx, j, d_times, d_mags, offsets, stream);
}

int pf_aov_dev(pf_ctx* ctx, const float* d_times, const float* d_mags, const int64_t* offsets,
               uint64_t n_curves, const float* d_periods, uint64_t n_per, const float* d_pdts,
               uint64_t n_pdt, uint32_t n_phase, uint32_t phase_overlap, int mode, float* d_out,
               void* stream) {
    Job j;
    j.algo = ALGO_AOV;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = d_periods;
    j.n_per = n_per;
    j.pdts = d_pdts;
    j.n_pdt = n_pdt;
    j.n_phase = n_phase;
    j.po = phase_overlap;
    j.out = d_out;
    return run_dev(ctx, j, d_times, d_mags, offsets, stream);
}

int pf_ls_dev(pf_ctx* ctx, const float* d_times, const float* d_mags, const int64_t* offsets,
              uint64_t n_curves, const float* d_periods, uint64_t n_per, const float* d_pdts,
              uint64_t n_pdt, int mode, float* d_out, void* stream) {
    Job j;
    j.algo = ALGO_LS;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = d_periods;
    j.n_per = n_per;
    j.pdts = d_pdts;
    j.n_pdt = n_pdt;
    j.out = d_out;
    return run_dev(ctx, j, d_times, d_mags, offsets, stream);
}

int pf_find_peaks_dev(pf_ctx* ctx, const float* d_data, uint64_t n_curves, uint64_t flat_len,
                      uint32_t n_peaks, uint32_t min_distance, int use_max, int64_t* d_out_idx,
                      float* d_out_val, void* stream) {
    if (!ctx) return PF_EINVAL;
    if (n_curves == 0 || n_peaks == 0) return PF_OK;
    if (!d_data || !d_out_idx || !d_out_val) return fail(ctx, PF_EINVAL, "NULL argument");
    if (n_curves > 0x7FFFFFFFull) return fail(ctx, PF_EINVAL, "too many curves");
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;  // NULL: the CUDA default stream
    PF_CUDA(launch_peaks(d_data, n_curves, flat_len, n_peaks, min_distance, use_max, d_out_idx,
                         d_out_val, s),
            "peak kernel launch");
    ctx->launches++;
    return PF_OK;
}

// ------------------------------------------------------------- batch plans

}  // extern "C"

struct pf_plan {
    pf_ctx* ctx = nullptr;  // private: its buffers and staging belong to the plan
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

struct PlanArgs {
    Job j;
    const float* d_times;
    const float* d_mags;
    std::vector<int64_t> offsets;
    uint32_t n_peaks, min_distance;
    int64_t* d_peak_idx;
    float* d_peak_val;
};

// The plan's work on `s`: the device-pointer pipeline, then the peak search.
int plan_enqueue(pf_ctx* ctx, const PlanArgs& a, cudaStream_t s) {
    int rc = run_dev(ctx, a.j, a.d_times, a.d_mags, a.offsets.data(), s);
    if (rc != PF_OK) return rc;
    if (a.n_peaks > 0 && a.j.n_curves > 0 && a.j.n_per * a.j.n_pdt > 0) {
        PF_CUDA(launch_peaks(a.j.out, a.j.n_curves, a.j.n_per * a.j.n_pdt, a.n_peaks,
                             a.min_distance, a.j.algo == ALGO_CE ? 0 : 1, a.d_peak_idx,
                             a.d_peak_val, s),
                "peak kernel launch");
        ctx->launches++;
    }
    return PF_OK;
}

}  // namespace

extern "C" {

int pf_plan_create(int device, int algo, const float* d_times, const float* d_mags,
                   const int64_t* offsets, uint64_t n_curves, const float* d_periods,
                   uint64_t n_per, const float* d_pdts, uint64_t n_pdt, uint32_t n_phase,
                   uint32_t n_mag, uint32_t phase_overlap, uint32_t mag_overlap, int mode,
                   float* d_out, uint32_t n_peaks, uint32_t min_distance, int64_t* d_peak_idx,
                   float* d_peak_val, pf_plan** out) {
    if (!out) return PF_EINVAL;
    *out = nullptr;
    if (algo != PF_ALGO_CE && algo != PF_ALGO_AOV && algo != PF_ALGO_LS) {
        g_create_error = "algo must be PF_ALGO_CE, PF_ALGO_AOV or PF_ALGO_LS";
        return PF_EINVAL;
    }
    if (mode & PF_TIMING) {
        g_create_error = "PF_TIMING is not available in a plan";
        return PF_EINVAL;
    }
    if (!offsets || !d_out || (n_peaks > 0 && (!d_peak_idx || !d_peak_val))) {
        g_create_error = "NULL argument";
        return PF_EINVAL;
    }
    PlanArgs a;
    a.j.algo = algo == PF_ALGO_CE ? ALGO_CE : algo == PF_ALGO_AOV ? ALGO_AOV : ALGO_LS;
    a.j.mode = mode;
    a.j.n_curves = n_curves;
    a.j.periods = d_periods;
    a.j.n_per = n_per;
    a.j.pdts = d_pdts;
    a.j.n_pdt = n_pdt;
    a.j.n_phase = n_phase;
    a.j.n_mag = n_mag;
    a.j.po = phase_overlap;
    a.j.mo = mag_overlap;
    a.j.out = d_out;
    a.d_times = d_times;
    a.d_mags = d_mags;
    a.offsets.assign(offsets, offsets + n_curves + 1);
    a.n_peaks = n_peaks;
    a.min_distance = min_distance;
    a.d_peak_idx = d_peak_idx;
    a.d_peak_val = d_peak_val;

    pf_plan* plan = new pf_plan();
    int rc = pf_ctx_create(&plan->ctx, device);
    if (rc != PF_OK) {
        delete plan;
        return rc;
    }
    pf_ctx* ctx = plan->ctx;
    auto bail = [&](int code) {
        g_create_error = ctx->err;
        pf_plan_destroy(plan);
        return code;
    };
    // Eager pass: tunes the launch shapes, sizes every buffer, loads kernels.
    cudaStream_t s = ctx->stream;
    if ((rc = plan_enqueue(ctx, a, s)) != PF_OK) return bail(rc);
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "plan warm-up"));
    ctx->staged_pending = false;
    ctx->done_recorded = false;
    ctx->timed_pending = false;
    // Captured pass: the same calls find the tuned shapes and sized buffers,
    // so nothing allocates or synchronises while the stream is captured.
    if ((e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return bail(cuda_fail(ctx, e, "begin capture"));
    rc = plan_enqueue(ctx, a, s);
    e = cudaStreamEndCapture(s, &plan->graph);
    ctx->staged_pending = false;
    ctx->done_recorded = false;
    ctx->timed_pending = false;
    if (rc != PF_OK) return bail(rc);
    if (e != cudaSuccess) return bail(cuda_fail(ctx, e, "end capture"));
    if ((e = cudaGraphInstantiate(&plan->exec, plan->graph, 0)) != cudaSuccess)
        return bail(cuda_fail(ctx, e, "graph instantiate"));
    *out = plan;
    return PF_OK;
}

int pf_plan_launch(pf_plan* plan, void* stream) {
    if (!plan || !plan->exec) return PF_EINVAL;
    pf_ctx* ctx = plan->ctx;
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    PF_CUDA(cudaGraphLaunch(plan->exec, (cudaStream_t)stream), "graph launch");
    return PF_OK;
}

const char* pf_plan_error(const pf_plan* plan) {
    return plan ? plan->ctx->err.c_str() : g_create_error.c_str();
}

void pf_plan_destroy(pf_plan* plan) {
    if (!plan) return;
    if (plan->ctx) cudaSetDevice(plan->ctx->device);
    if (plan->exec) cudaGraphExecDestroy(plan->exec);
    if (plan->graph) cudaGraphDestroy(plan->graph);
    if (plan->ctx) pf_ctx_destroy(plan->ctx);
    delete plan;
}

uint64_t pf_plan_kernel_count(const pf_plan* plan) {
    if (!plan || !plan->graph) return 0;
    size_t n = 0;
    if (cudaGraphGetNodes(plan->graph, nullptr, &n) != cudaSuccess) return 0;
    std::vector<cudaGraphNode_t> nodes(n);
    if (n && cudaGraphGetNodes(plan->graph, nodes.data(), &n) != cudaSuccess) return 0;
    uint64_t k = 0;
    for (size_t i = 0; i < n; i++) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nodes[i], &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
    }
    return k;
}

int pf_ce_stats(pf_ctx* ctx, const float* const* times, const float* const* mags,
                const uint64_t* lengths, uint64_t n_curves, const float* periods,
                uint64_t n_per, const float* period_dts, uint64_t n_pdt, uint32_t n_phase,
                uint32_t n_mag, uint32_t phase_overlap, uint32_t mag_overlap, uint32_t n_top,
                int mode, float* out_stats, int64_t* out_idx, float* out_val) {
    Job j;
    j.algo = ALGO_CE;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = periods;
    j.n_per = n_per;
    j.pdts = period_dts;
    j.n_pdt = n_pdt;
    j.n_phase = n_phase;
    j.n_mag = n_mag;
    j.po = phase_overlap;
    j.mo = mag_overlap;
    j.stats = true;
    j.n_top = n_top;
    j.out_stats = out_stats;
    j.out_idx = out_idx;
    j.out_val = out_val;
    return run_host(ctx, j, times, mags, lengths);
}

int pf_aov_stats(pf_ctx* ctx, const float* const* times, const float* const* mags,
                 const uint64_t* lengths, uint64_t n_curves, const float* periods,
                 uint64_t n_per, const float* period_dts, uint64_t n_pdt, uint32_t n_phase,
                 uint32_t phase_overlap, uint32_t n_top, int mode, float* out_stats,
                 int64_t* out_idx, float* out_val) {
    Job j;
    j.algo = ALGO_AOV;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = periods;
    j.n_per = n_per;
    j.pdts = period_dts;
    j.n_pdt = n_pdt;
    j.n_phase = n_phase;
    j.po = phase_overlap;
    j.stats = true;
    j.n_top = n_top;
    j.out_stats = out_stats;
    j.out_idx = out_idx;
    j.out_val = out_val;
    return run_host(ctx, j, times, mags, lengths);
}

int pf_ls_stats(pf_ctx* ctx, const float* const* times, const float* const* mags,
                const uint64_t* lengths, uint64_t n_curves, const float* periods,
                uint64_t n_per, const float* period_dts, uint64_t n_pdt, uint32_t n_top,
                int mode, float* out_stats, int64_t* out_idx, float* out_val) {
    Job j;
    j.algo = ALGO_LS;
    j.mode = mode;
    j.n_curves = n_curves;
    j.periods = periods;
    j.n_per = n_per;
    j.pdts = period_dts;
    j.n_pdt = n_pdt;
    j.stats = true;
    j.n_top = n_top;
    j.out_stats = out_stats;
    j.out_idx = out_idx;
    j.out_val = out_val;
    return run_host(ctx, j, times, mags, lengths);
}

int pf_find_peaks(pf_ctx* ctx, const float* data, uint64_t n_curves, uint64_t flat_len,
                  uint32_t n_peaks, uint32_t min_distance, int use_max, int64_t* out_idx,
                  float* out_val) {
    if (!ctx) return PF_EINVAL;
    if (n_curves == 0 || n_peaks == 0) return PF_OK;
    if (!data || !out_idx || !out_val) return fail(ctx, PF_EINVAL, "NULL argument");
    if (n_curves > 0x7FFFFFFFull) return fail(ctx, PF_EINVAL, "too many curves");
    PF_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const size_t in_bytes = (size_t)n_curves * flat_len * 4;
    const size_t pk = (size_t)n_curves * n_peaks;
    int rc = ensure_dev(ctx, ctx->d_out, in_bytes);
    if (rc != PF_OK) return rc;
    if ((rc = ensure_dev(ctx, ctx->d_pidx, pk * 8)) != PF_OK) return rc;
    if ((rc = ensure_dev(ctx, ctx->d_pval, pk * 4)) != PF_OK) return rc;
    cudaStream_t s = ctx->stream;
    if ((rc = order_after_previous(ctx, s)) != PF_OK) return rc;
    PF_CUDA(cudaMemcpyAsync(ctx->d_out.p, data, in_bytes, cudaMemcpyHostToDevice, s), "H2D");
    PF_CUDA(launch_peaks((const float*)ctx->d_out.p, n_curves, flat_len, n_peaks, min_distance,
                         use_max, (int64_t*)ctx->d_pidx.p, (float*)ctx->d_pval.p, s),
            "peak kernel launch");
    ctx->launches++;
    PF_CUDA(cudaMemcpyAsync(out_idx, ctx->d_pidx.p, pk * 8, cudaMemcpyDeviceToHost, s), "D2H");
    PF_CUDA(cudaMemcpyAsync(out_val, ctx->d_pval.p, pk * 4, cudaMemcpyDeviceToHost, s), "D2H");
    if ((rc = mark_done(ctx, s)) != PF_OK) return rc;
    PF_CUDA(cudaStreamSynchronize(s), "stream synchronize");
    return PF_OK;
}

}  // extern "C"
