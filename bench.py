"""Benchmark: curve x period x point evaluations per second on B200.

Default workload (one "step"): the mixed ragged batch -- 100 000 light
curves with lengths lognormal (median 300, sigma 0.8) clipped to [20, 2000]
(4.07e7 points), seasonal cadence over 2500 days, a third sinusoids, a third
box eclipses, a third pure noise -- searched by Conditional Entropy (10 x 10
bins), AOV (15 bins) and Lomb-Scargle over 20 000 log-spaced trial periods
in [0.05, 500] days (one period derivative, 0), each followed by the top-32
peak search: 3 x 8.14e11 evaluations per step.  Seeded synthetic curves with
the configuration's shapes (no public dataset is named by the reference).

Reported (one JSON line on rank 0):
  value       evals/s of the chosen form: per step, the magnitudes are
              prepared on the device (CE normalised, LS centred, numpy's
              values) and the three batch plans (CUDA graphs of the queue
              kernels per length class + peak search) are replayed; inputs
              resident in HBM, CUDA events around each step, max over ranks.
  plain       the same step with the plain form (the reference's fold op for
              op, one launch per algorithm) and its ratio chosen / plain.
  e2e         the same metric through the C ABI with host buffers: per step
              host magnitude preparation, pf_{ce,aov,ls}_peaks from per-curve
              host arrays (H2D copy of every curve inside each call), peaks
              back to host memory; the calls are pipelined (PF_ASYNC).
  e2e_calc    once per algorithm (after a warm-up call on 30% of the
              curves), the public Python path calc(list of numpy,
              output='peaks'), which also builds the 3.2e6 result objects
              per algorithm.
  latency     per-curve device latency p50 / p99 (PF_TIMING stamps), chosen
              and plain.
  roofline    the kernel with the most time in the step, against the
              measured rate of the pipe that bounds it (pipe_peaks.cu probe).
  ls_peak_frequency_error  Newton-refined LS peaks of the chosen form on a
              sample of curves, checked by one FP64 Newton step.
  cpu_baseline / reference_cuda  the C/OpenMP restatement of the reference's
              Rust CPU path on the host cores, and the reference's own CUDA
              drivers built from its sources, each on a stated curve sample.
  batch_4096  secondary: CE(10x10) + AOV(15) + peaks over 1000 curves x 4096
              points x 10000 periods x pdts [0, 1e-6], chosen vs plain.

--impl reference runs the CPU restatement of the reference's path (the
reference's CPU implementation is Rust; no Rust toolchain exists on these
machines) as the reference arm, on rank 0 only.  --workload selects the
separate reports of the other configurations (bench_reports.py).
"""

from __future__ import annotations

import argparse
import contextlib
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import lightcurves as lc  # noqa: E402

METRIC = "curve*period*point evals/s on 1 B200, chosen vs plain, at stated error"
SEED = 20261205
N_PEAKS = 32
ALGOS = ("ce", "aov", "ls")

# The mixed ragged batch.
RAGGED_CURVES = 100000
RAGGED_PERIODS = 20000
RAGGED_WORKLOAD = ("mixed ragged batch: 100000 curves, lengths lognormal(median 300, sigma 0.8) "
                   "clipped to [20, 2000], seasonal cadence 2500 d, 1/3 sinusoid, 1/3 box "
                   "eclipse, 1/3 noise; CE(10x10) + AOV(15) + LS over 20000 log periods "
                   "[0.05, 500] d, period_dts [0], top-32 peaks each")

# The 1000 x 4096 batch (secondary line; --workload batch / fpw / bls / device).
N_CURVES = 1000
N_POINTS = 4096
N_PERIODS = 10000
PDTS = (0.0, 1e-6)


def ragged_grid():
    periods = np.exp(np.linspace(np.log(0.05), np.log(500.0), RAGGED_PERIODS)).astype(np.float32)
    return periods, np.zeros(1, np.float32)


def make_workload(n_curves=N_CURVES, seed=SEED):
    ts, ms = lc.mixed_signal_batch(n_curves, N_POINTS, seed)
    periods = np.exp(np.linspace(np.log(0.1), np.log(100.0), N_PERIODS)).astype(np.float32)
    return ts, ms, periods, np.array(PDTS, np.float32)


# ----------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi samples (200 ms) while a timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.idx)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (FileNotFoundError, OSError):
            self.proc = None
            return self
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"],
                    "samples": 0}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        return summarise_clocks(self.lines)


def summarise_clocks(lines):
    """Median SM clock, max clock, throttle reasons seen active, samples."""
    mhz, mx, reasons, power = [], None, set(), []
    for ln in lines:
        parts = [p.strip() for p in ln.split(",")]
        if len(parts) < 9:
            continue
        try:
            mhz.append(float(parts[1]))
            mx = float(parts[2])
            power.append(float(parts[3]))
        except ValueError:
            continue
        for nm, v in zip(ClockSampler.REASONS, parts[5:9]):
            if v.lower() == "active":
                reasons.add(nm)
    return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
            "reasons": sorted(reasons), "samples": len(mhz),
            "power_w_max": max(power) if power else None}


class Clocks:
    """A clock record per timed region (one nvidia-smi sampler each) and
    their union."""

    def __init__(self, device_index):
        self.idx = device_index
        self.regions = {}
        self._lines = []

    @contextlib.contextmanager
    def region(self, name):
        s = ClockSampler(self.idx).start()
        try:
            yield
        finally:
            self.regions[name] = s.stop()
            self._lines.extend(s.lines)

    def union(self):
        return summarise_clocks(self._lines)


# -------------------------------------------------------------- pipe peaks


def measure_pipes():
    """Per-pipe throughput measured now on this GPU (pipe_peaks.cu beside
    this file, built on first use): the roofline denominators."""
    so = os.path.join(ROOT, "pipe_peaks.so")
    src = os.path.join(ROOT, "pipe_peaks.cu")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        from periodfind_b200.build import ARCH, COMMON, nvcc

        subprocess.run([nvcc()] + COMMON + ARCH + ["-shared", "-o", so, src], check=True)
    lib = ctypes.CDLL(so)

    class R(ctypes.Structure):
        _fields_ = [("name", ctypes.c_char * 32), ("ops_per_clk_per_sm", ctypes.c_double),
                    ("ops_per_s", ctypes.c_double), ("sm_mhz", ctypes.c_double)]

    arr = (R * 32)()
    k = lib.pfpk_measure(0, arr, 32)
    return {arr[i].name.decode(): {"per_s": arr[i].ops_per_s,
                                   "per_clk_sm": arr[i].ops_per_clk_per_sm,
                                   "mhz": arr[i].sm_mhz} for i in range(max(k, 0))}


# The pipe that bounds each kernel of the ragged step, and its algorithmic
# operations per evaluation (no period derivative):
#   CE bin kernel   FP64: t * RN(1/P) (DMUL), floor (DADD.RD), bin with
#                   fraction bits (DFMA.RD); one shared reduction.
#   AOV bin kernel  two shared reductions (count, fixed-point sum); 3 FP64.
#   LS fold kernel  MUFU sine and cosine.
ROOFLINE = {
    # Operations the chosen kernels perform per evaluation: CE one shared
    # u32 reduction (its 16-bit counter) and one FP64 FMA; AOV two
    # reductions (count, fixed-point sum) and one FP64 FMA; LS a MUFU sine
    # and cosine.  (Without a period derivative, |q| < 2^19.)
    "ce": {"kernel": "bin_kernel<CE> (chosen)", "bound": "shared-atomic",
           "pipe": "atoms_u32_private", "ops": 1.0, "views": {"fp64": ("dfma", 1.0)}},
    "aov": {"kernel": "bin_kernel<AOV> (chosen)", "bound": "shared-atomic",
            "pipe": "atoms_u32_private", "ops": 2.0, "views": {"fp64": ("dfma", 1.0)}},
    "ls": {"kernel": "fold_kernel<LS, split-precision> (chosen)", "bound": "mufu",
           "pipe": "mufu_sin+cos", "ops": 2.0, "views": {}},
}
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the class
# kernels of one call over the whole ragged batch: one ncu capture of a
# 3000-curve sample of the batch (bench.py --workload profile --curves 3000),
# scaled by its evaluations (x 32.64; the traffic is the curve points read
# and the periodogram written, both proportional).
RAGGED_TRAFFIC = {"ce": 3.82e9, "aov": 3.90e9, "ls": 3.62e9}


# ------------------------------------------------------------ ragged step


class RaggedStep:
    """The ragged batch resident on the device, its three batch plans
    (chosen) and the plain form's direct calls, on the current stream."""

    def __init__(self, t, m, off, periods, pdts, torch, device, plans=True):
        from periodfind_b200 import _native as nat
        from periodfind_b200.plan import BatchPlan

        self.nat, self.torch = nat, torch
        self.off = np.ascontiguousarray(off, np.int64)
        self.n = len(off) - 1
        dev = torch.device("cuda", device)
        self.d_t = torch.from_numpy(t).to(dev)
        self.d_m = torch.from_numpy(m).to(dev)
        self.mags = {"ce": torch.empty_like(self.d_m), "aov": self.d_m,
                     "ls": torch.empty_like(self.d_m)}
        self.d_p = torch.from_numpy(periods).to(dev)
        self.d_d = torch.from_numpy(pdts).to(dev)
        self.n_per, self.n_pdt = len(periods), len(pdts)
        self.cells = self.n_per * self.n_pdt
        self.pg = torch.empty((self.n, self.cells), dtype=torch.float32, device=dev)
        self.pk_i = torch.empty((3, self.n, N_PEAKS), dtype=torch.int64, device=dev)
        self.pk_v = torch.empty((3, self.n, N_PEAKS), dtype=torch.float32, device=dev)
        # Magnitude preparation and the plain calls each on a context of
        # their own (a context serialises the reuse of its offsets copy).
        self.prep_ctx = {k: nat.Context(device) for k in ("ce", "ls")}
        self.ctx = nat.Context(device)
        self.stream = torch.cuda.current_stream(dev)
        self.s = self.stream.cuda_stream
        self.prepare()
        self.plans = {}
        for k, algo in enumerate(ALGOS if plans else ()):
            self.plans[algo] = BatchPlan(
                algo, self.d_t, self.mags[algo], self.off, self.d_p, self.d_d, self.pg,
                n_phase=10 if algo == "ce" else 15, n_mag=10, flags=nat.PF_MODE_CHOSEN,
                n_peaks=N_PEAKS, peak_idx=self.pk_i[k], peak_val=self.pk_v[k], device=device)
        self.plan_kernels = sum(int(nat.load().pf_plan_kernel_count(p.handle))
                                for p in self.plans.values())

    def prepare(self):
        nat = self.nat
        for algo, kind in (("ce", nat.PF_PREP_NORMALIZE), ("ls", nat.PF_PREP_CENTER)):
            c = self.prep_ctx[algo]
            c.check(c.lib.pf_prepare_mags_dev(c.handle, self.d_m.data_ptr(), self.off.ctypes.data,
                                              self.n, kind, self.mags[algo].data_ptr(), self.s))

    def chosen(self):
        self.prepare()
        for algo in ALGOS:
            self.plans[algo].launch(self.stream)

    def direct(self, algo, flags, peaks=True):
        c, lib, h = self.ctx, self.ctx.lib, self.ctx.handle
        common = (h, self.d_t.data_ptr(), self.mags[algo].data_ptr(), self.off.ctypes.data,
                  self.n, self.d_p.data_ptr(), self.n_per, self.d_d.data_ptr(), self.n_pdt)
        if algo == "ce":
            c.check(lib.pf_ce_dev(*common, 10, 10, 1, 1, flags, self.pg.data_ptr(), self.s))
        elif algo == "aov":
            c.check(lib.pf_aov_dev(*common, 15, 1, flags, self.pg.data_ptr(), self.s))
        else:
            c.check(lib.pf_ls_dev(*common, flags, self.pg.data_ptr(), self.s))
        if peaks:
            k = ALGOS.index(algo)
            c.check(lib.pf_find_peaks_dev(h, self.pg.data_ptr(), self.n, self.cells, N_PEAKS, 1,
                                          0 if algo == "ce" else 1, self.pk_i[k].data_ptr(),
                                          self.pk_v[k].data_ptr(), self.s))

    def plain(self):
        self.prepare()
        for algo in ALGOS:
            self.direct(algo, self.nat.PF_MODE_PLAIN)

    def close(self):
        for p in self.plans.values():
            p.close()


def time_steps(fn, steps, warmup, torch, flush, stream):
    """Mean CUDA-event time (ms) of `steps` calls of fn after `warmup`
    untimed ones; L2 flushed (a 256 MB write) before each timed call,
    outside the events."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    per = []
    for _ in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        per.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    return float(np.mean(per)), per


def curve_latency(step, algo, flags):
    """Per-curve device latency (ms) of one stamped direct call: last end
    minus first start of the CTAs that computed the curve."""
    nat = step.nat
    step.direct(algo, flags | nat.PF_TIMING, peaks=False)
    lat = np.zeros(step.n)
    step.ctx.check(step.ctx.lib.pf_curve_latency(step.ctx.handle, step.n, lat.ctypes.data))
    return {"p50_ms": float(np.percentile(lat, 50)) / 1e6,
            "p99_ms": float(np.percentile(lat, 99)) / 1e6}


# ---------------------------------------------------------- end to end


class HostBatch:
    """The ragged batch as per-curve host arrays (views of two flat float32
    arrays) with the per-curve pointers the C ABI takes."""

    def __init__(self, t, m, off):
        self.t, self.m, self.off = t, m, off
        self.n = len(off) - 1
        self.lens = np.diff(off).astype(np.uint64)
        self.tptr = self.ptrs(t)
        self.mptr = self.ptrs(m)

    def ptrs(self, a):
        return (np.uint64(a.ctypes.data)
                + np.uint64(4) * self.off[:-1].astype(np.uint64)).astype(np.uintp)


def e2e_cabi(hb, periods, pdts, steps, warmup, device):
    """Wall time per step of CE + AOV + LS peaks through the C ABI from host
    buffers: the peak calls -- each packs its curves into pinned staging
    with the magnitude preparation (PF_HOST_NORMALIZE / PF_HOST_CENTER),
    copies them to the GPU, runs the kernels and the peak search and copies
    the peaks back -- pipelined with PF_ASYNC so that host work overlaps the
    GPU.  Returns (s per step, H2D bytes, D2H bytes, kernel launches per
    step)."""
    from periodfind_b200 import _native as nat

    ctx = nat.Context(device)
    lib, h = ctx.lib, ctx.handle
    n = hb.n
    idx = np.empty((3, n, N_PEAKS), np.int64)
    val = np.empty((3, n, N_PEAKS), np.float32)
    flags = nat.PF_MODE_CHOSEN | nat.PF_ASYNC
    grid = (periods.ctypes.data, len(periods), pdts.ctypes.data, len(pdts))

    def peaks(algo, k, a, e, prep):
        # Curves [a, e): pointers, lengths and output rows from offset a.
        ptr = lambda arr, itemsize: arr.ctypes.data + a * itemsize
        args = (h, ptr(hb.tptr, 8), ptr(hb.mptr, 8), ptr(hb.lens, 8), e - a) + grid
        out = (flags | prep, ptr(idx[k], 8 * N_PEAKS), ptr(val[k], 4 * N_PEAKS))
        if algo == "ce":
            rc = lib.pf_ce_peaks(*args, 10, 10, 1, 1, N_PEAKS, 1, *out)
        elif algo == "aov":
            rc = lib.pf_aov_peaks(*args, 15, 1, N_PEAKS, 1, *out)
        else:
            rc = lib.pf_ls_peaks(*args, N_PEAKS, 1, *out)
        ctx.check(rc)

    q = n // 4

    def step():
        # The magnitudes are normalised (CE) or centred (LS) as they are
        # packed (numpy's values).  CE goes in two calls, a quarter of the
        # curves first, so that the GPU starts once that quarter is packed;
        # each later call is packed while the GPU runs the one before.
        peaks("ce", 0, 0, q, nat.PF_HOST_NORMALIZE)
        peaks("ce", 0, q, n, nat.PF_HOST_NORMALIZE)
        ctx.check(lib.pf_wait(h))
        peaks("aov", 1, 0, n, 0)
        ctx.check(lib.pf_wait(h))
        peaks("ls", 2, 0, n, nat.PF_HOST_CENTER)
        ctx.check(lib.pf_wait(h))
        ctx.check(lib.pf_wait(h))

    for _ in range(warmup):
        step()
    l0 = ctx.launches
    w = []
    for _ in range(steps):
        t0 = time.perf_counter()
        step()
        w.append(time.perf_counter() - t0)
    launches = (ctx.launches - l0) // max(steps, 1)
    h2d = 3 * (hb.t.nbytes + hb.m.nbytes + periods.nbytes + pdts.nbytes)
    d2h = idx.nbytes + val.nbytes
    ctx.close()
    return float(np.mean(w)), int(h2d), int(d2h), int(launches)


def e2e_calc(t, m, off, periods, pdts, device):
    """Seconds of one calc(list of numpy arrays, output='peaks') per
    algorithm through the public Python classes (result objects built),
    after a warm-up call on the first 30% of the curves (the context's
    tuning for each length class and its pinned staging, as a long-running
    caller would have them)."""
    from periodfind_b200 import gpu

    ts, ms = lc.split_csr(t, off), lc.split_csr(m, off)
    k = max(1, (3 * len(ts)) // 10)
    out = {}
    for algo, obj in (("ce", gpu.ConditionalEntropy(10, 10, device=device)),
                      ("aov", gpu.AOV(15, device=device)),
                      ("ls", gpu.LombScargle(device=device))):
        obj.calc(ts[:k], ms[:k], periods, pdts, output="peaks", n_peaks=N_PEAKS)
        t0 = time.perf_counter()
        res = obj.calc(ts, ms, periods, pdts, output="peaks", n_peaks=N_PEAKS)
        out[algo] = time.perf_counter() - t0
        assert len(res) == len(ts)
        del res
    return out


# ------------------------------------------------------- LS peak precision


def _ls_derivs_f64(t, y, w):
    """LS power P and its first and second derivatives in the angular
    frequency, FP64, for one curve (times t measured from their span's
    midpoint) at the frequencies w.  P = 0.5 v^T M^-1 v with v = (sum y cos,
    sum y sin) and M the normal matrix of (cos, sin) -- the reference's
    tau-rotated power (periodfind/cuda/ls.cu:107-134) in closed form; with
    w_ = M^-1 v and u = v' - M' w_:  P' = w_.v' - 0.5 w_^T M' w_,
    P'' = u^T M^-1 u + w_.v'' - 0.5 w_^T M'' w_."""
    th = np.outer(w, t)
    c, s = np.cos(th), np.sin(th)
    t1, t2 = t, t * t
    v = np.stack([c @ y, s @ y], -1)
    v1 = np.stack([-(s * t1) @ y, (c * t1) @ y], -1)
    v2 = np.stack([-(c * t2) @ y, -(s * t2) @ y], -1)
    cc, cs, ss = (c * c).sum(1), (c * s).sum(1), (s * s).sum(1)
    d1 = ((c * c - s * s) * t1).sum(1)
    x1 = ((c * s) * t1).sum(1)
    d2 = ((c * c - s * s) * t2).sum(1)
    x2 = ((c * s) * t2).sum(1)

    def mat(a, b, d):
        return np.stack([np.stack([a, b], -1), np.stack([b, d], -1)], -2)

    M = mat(cc, cs, ss)
    M1 = mat(-2 * x1, d1, 2 * x1)
    M2 = mat(-2 * d2, -4 * x2, 2 * d2)
    Mi = np.linalg.inv(M)
    wv = np.einsum("kij,kj->ki", Mi, v)
    P = 0.5 * np.einsum("ki,ki->k", wv, v)
    q1 = np.einsum("ki,kij,kj->k", wv, M1, wv)
    P1 = np.einsum("ki,ki->k", wv, v1) - 0.5 * q1
    u = v1 - np.einsum("kij,kj->ki", M1, wv)
    P2 = (np.einsum("ki,kij,kj->k", u, Mi, u) + np.einsum("ki,ki->k", wv, v2)
          - 0.5 * np.einsum("ki,kij,kj->k", wv, M2, wv))
    return P, P1, P2


def _refine_f64(t, y, w0, hw, n_steps=5, keep_last=1e-5):
    """The GPU's safeguarded Newton refinement (pf_ls_refine_dev) in FP64:
    Newton where P'' < 0, otherwise a quarter-bracket step uphill, every
    iterate clamped to [w0 - hw, w0 + hw]; the last iterate unless its power
    is more than keep_last below the best."""
    w = w0.copy()
    best_w, best_p = w.copy(), np.full_like(w, -1.0)
    last_w, last_p = w.copy(), best_p.copy()
    moved = np.full_like(w, np.inf)
    for e in range(n_steps + 1):
        P, P1, P2 = _ls_derivs_f64(t, y, w)
        last_w, last_p = w.copy(), P
        up = P > best_p
        best_w = np.where(up, w, best_w)
        best_p = np.where(up, P, best_p)
        if e < n_steps:
            step = np.where(P2 < 0, -P1 / np.where(P2 < 0, P2, -1.0),
                            np.where(P1 > 0, 0.25 * hw, -0.25 * hw))
            nw = np.clip(w + step, w0 - hw, w0 + hw)
            moved = np.abs(nw - w) / np.abs(w)
            w = nw
    out = np.where(last_p >= best_p * (1.0 - keep_last), last_w, best_w)
    return out, moved


def ls_peak_error(step, periods, n_sample, torch, seed=SEED + 9):
    """Refine the chosen LS periodogram's top-32 grid peaks of a random sample
    of curves by 5 Newton steps on the GPU (pf_ls_refine_dev), and the same
    peaks by the same iteration in FP64 (numpy) from the same starts: the
    relative difference of the refined frequencies is the error of the
    GPU's FP32 sums and split-precision phases against FP64."""
    from periodfind_b200 import ls_grad

    rng = np.random.default_rng(seed)
    cur = np.sort(rng.choice(step.n, n_sample, replace=False))
    idx = step.pk_i[2].cpu().numpy()[cur]
    off = step.off
    t_all = step.d_t.cpu().numpy()
    y_all = step.mags["ls"].cpu().numpy()
    ts = [t_all[off[c]:off[c + 1]] for c in cur]
    ys = [y_all[off[c]:off[c + 1]] for c in cur]
    sub_off = np.zeros(n_sample + 1, np.int64)
    np.cumsum([len(x) for x in ts], out=sub_off[1:])
    grid = 2.0 * np.pi / periods.astype(np.float64)
    valid = idx >= 0
    i = np.where(valid, idx, 0)
    w0 = grid[i]
    hw = np.maximum(np.abs(grid[np.maximum(i - 1, 0)] - w0),
                    np.abs(grid[np.minimum(i + 1, len(grid) - 1)] - w0))
    dev = step.d_t.device
    w, _ = ls_grad.refine_peaks(torch.from_numpy(np.concatenate(ts)).to(dev),
                                torch.from_numpy(np.concatenate(ys)).to(dev),
                                torch.from_numpy(w0).to(dev), torch.from_numpy(hw).to(dev),
                                sub_off, n_steps=5)
    w = w.cpu().numpy()
    errs, conv = [], []
    for k in range(n_sample):
        v = valid[k]
        if len(ts[k]) < 16 or not v.any():
            continue
        t = ts[k].astype(np.float64)
        t = t - 0.5 * (t.min() + t.max())
        ref, moved = _refine_f64(t, ys[k].astype(np.float64), w0[k][v], hw[k][v])
        errs.extend((np.abs(w[k][v] - ref) / ref).tolist())
        conv.extend((moved <= 1e-9).tolist())
    errs = np.array(errs) if errs else np.zeros(1)
    conv = np.array(conv, bool) if conv else np.ones(1, bool)
    ec = errs[conv] if conv.any() else np.zeros(1)
    return {"peaks": int(errs.size), "curves": n_sample,
            "converged_peaks": int(conv.sum()),
            "max_rel_converged": float(ec.max()), "median_rel": float(np.median(errs)),
            "p99_rel": float(np.percentile(errs, 99)), "max_rel_all": float(errs.max()),
            "within_target": float(np.mean(errs <= 1e-7)), "target": 1e-7,
            "method": "top-32 grid peaks of the chosen LS periodogram of 64 random curves, "
                      "refined by 5 safeguarded Newton steps on the GPU (pf_ls_refine_dev) and "
                      "by the same iteration in FP64 (numpy, analytic derivatives) from the "
                      "same starts; relative frequency difference.  'converged': the FP64 "
                      "iteration's last step moved the frequency by at most 1e-9 (elsewhere "
                      "the 5-step iteration has not settled and the difference measures the "
                      "path, not the arithmetic)"}


# ------------------------------------------------------------ baselines


def _sample_curves(off, k, seed):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(len(off) - 1, min(k, len(off) - 1), replace=False))


def _subset(t, m, off, cur):
    return ([t[off[c]:off[c + 1]] for c in cur], [m[off[c]:off[c + 1]] for c in cur])


def oracle_ragged(O, ts, ms, periods, pdts, cores):
    """CE + AOV + LS with peaks by the CPU restatement of the Rust path
    (rust/src/lib.rs:31-199, 508-677), magnitudes prepared as the
    reference's classes prepare them."""
    msn = [lc.normalize(m) for m in ms]
    msc = [lc.center(m) for m in ms]
    for pg, use_max in ((O.ce(ts, msn, periods, pdts, 10, 10, n_threads=cores), False),
                        (O.aov(ts, ms, periods, pdts, 15, n_threads=cores), True),
                        (O.ls(ts, msc, periods, pdts, n_threads=cores), True)):
        O.find_top_peaks_batched(pg, N_PEAKS, 1, use_max, n_threads=cores)


def cpu_baseline(t, m, off, periods, pdts, target_s=12.0):
    """The oracle on all host cores over a random sample of curves (the
    batch's length distribution) sized for about target_s of work."""
    from oracle import oracle as O

    cores = os.cpu_count() or 1
    cur = _sample_curves(off, 100, SEED + 7)
    ts, ms = _subset(t, m, off, cur)
    t0 = time.perf_counter()
    oracle_ragged(O, ts, ms, periods, pdts, cores)
    one = time.perf_counter() - t0
    k = int(max(50, min(len(off) - 1, 100 * target_s / max(one, 1e-3))))
    cur = _sample_curves(off, k, SEED + 7)
    ts, ms = _subset(t, m, off, cur)
    t0 = time.perf_counter()
    oracle_ragged(O, ts, ms, periods, pdts, cores)
    dt = time.perf_counter() - t0
    ev = 3 * sum(len(x) for x in ts) * len(periods) * len(pdts)
    return {"value": ev / dt, "unit": "evals/s", "cores": cores, "kind": "port",
            "sample": f"{len(cur)} random curves of {len(off) - 1} (CE + AOV + LS periodograms "
                      f"and top-32 peaks over the full 20000-period grid), {dt:.1f} s on "
                      f"{cores} threads; C/OpenMP restatement of the reference's Rust path"}


def reference_cuda(t, m, off, periods, pdts, clocks, n_sample=1000):
    """The reference's own CUDA drivers (CalcCEValsBatched, CalcAOVValsBatched,
    CalcLSBatched; periodfind/cuda/{ce,aov,ls}.cu) built from its sources,
    on a random curve sample of the batch: periodograms only (the
    reference's GPU path has no peak search), with its per-call device
    allocation, per-curve copies and launches, as its Python classes call
    it.  A reported comparator beside the plain form."""
    from oracle import oracle as O

    if not O.ref_available():
        return {"unavailable": "oracle/_ref/libpfref.so is not built"}
    cur = _sample_curves(off, n_sample, SEED + 8)
    ts, ms = _subset(t, m, off, cur)
    msn = [lc.normalize(x) for x in ms]
    msc = [lc.center(x) for x in ms]
    O.ref_cuda("ce", ts[:8], msn[:8], periods, pdts, n_phase=10, n_mag=10)  # load, warm up
    out = {}
    with clocks.region("reference_cuda"):
        for algo, mm, kw in (("ce", msn, {"n_phase": 10, "n_mag": 10}),
                             ("aov", ms, {"n_phase": 15}), ("ls", msc, {})):
            t0 = time.perf_counter()
            O.ref_cuda(algo, ts, mm, periods, pdts, **kw)
            out[algo] = time.perf_counter() - t0
    ev = sum(len(x) for x in ts) * len(periods) * len(pdts)
    return {"value": 3 * ev / sum(out.values()), "unit": "evals/s",
            "per_algo_evals_per_s": {a: ev / s for a, s in out.items()},
            "sample": f"{len(cur)} random curves of {len(off) - 1}, full grid, wall time of the "
                      "reference's Calc*Batched host drivers, periodograms only",
            "clocks": clocks.regions.get("reference_cuda")}


def reference_arm(args):
    """The reference arm: the CPU restatement of the reference's Rust path on
    all host cores, each step a fixed random sample of the ragged batch."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O

    n_curves = args.curves or RAGGED_CURVES
    t, m, off = lc.ragged_batch(n_curves, SEED + 5)
    periods, pdts = ragged_grid()
    cores = os.cpu_count() or 1
    k = 60
    cur = _sample_curves(off, k, SEED + 7)
    ts, ms = _subset(t, m, off, cur)
    ev = 3 * sum(len(x) for x in ts) * len(periods) * len(pdts)
    for _ in range(args.warmup):
        oracle_ragged(O, ts, ms, periods, pdts, cores)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        oracle_ragged(O, ts, ms, periods, pdts, cores)
        times.append(time.perf_counter() - t0)
    per_step = float(np.mean(times))
    value = ev / per_step
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "evals/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 fold, f32 statistics", "data": "synthetic",
        "config": {"workload": RAGGED_WORKLOAD, "sample_curves_per_step": k},
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": cores, "kind": "port",
                         "sample": f"{k} random curves of {n_curves} per step (CE + AOV + LS "
                                   "periodograms and top-32 peaks, full grid); C/OpenMP "
                                   "restatement of the reference's Rust CPU path"},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------- 1000 x 4096 secondary


class BatchStep:
    """CE + AOV + peaks on the device-resident 1000 x 4096 batch."""

    def __init__(self, ts, ms, periods, pdts, flags, torch, device):
        from periodfind_b200 import _native as nat

        self.ctx = nat.Context(device)
        self.flags = flags
        off = np.zeros(len(ts) + 1, np.int64)
        np.cumsum([len(t) for t in ts], out=off[1:])
        self.off = off
        dev = torch.device("cuda", device)
        self.t = torch.from_numpy(np.concatenate(ts)).to(dev)
        self.m_ce = torch.from_numpy(np.concatenate([lc.normalize(m) for m in ms])).to(dev)
        self.m_aov = torch.from_numpy(np.concatenate(ms)).to(dev)
        self.P = torch.from_numpy(periods).to(dev)
        self.D = torch.from_numpy(pdts).to(dev)
        self.n = len(ts)
        self.cells = len(periods) * len(pdts)
        self.pg = torch.empty((2, self.n, self.cells), dtype=torch.float32, device=dev)
        self.pk_i = torch.empty((2, self.n, N_PEAKS), dtype=torch.int64, device=dev)
        self.pk_v = torch.empty((2, self.n, N_PEAKS), dtype=torch.float32, device=dev)
        self.np_, self.nd = len(periods), len(pdts)
        self.s = torch.cuda.current_stream(dev).cuda_stream

    def run(self):
        c, lib, h = self.ctx, self.ctx.lib, self.ctx.handle
        for k, m in enumerate((self.m_ce, self.m_aov)):
            common = (h, self.t.data_ptr(), m.data_ptr(), self.off.ctypes.data, self.n,
                      self.P.data_ptr(), self.np_, self.D.data_ptr(), self.nd)
            if k == 0:
                c.check(lib.pf_ce_dev(*common, 10, 10, 1, 1, self.flags, self.pg[0].data_ptr(),
                                      self.s))
            else:
                c.check(lib.pf_aov_dev(*common, 15, 1, self.flags, self.pg[1].data_ptr(),
                                       self.s))
            c.check(lib.pf_find_peaks_dev(h, self.pg[k].data_ptr(), self.n, self.cells, N_PEAKS,
                                          1, k, self.pk_i[k].data_ptr(), self.pk_v[k].data_ptr(),
                                          self.s))


def batch_secondary(torch, device, flush, clocks, steps=3):
    """The 1000 x 4096 batch: chosen and plain device steps (CUDA events, L2
    flushed between steps)."""
    from periodfind_b200 import _native as nat

    ts, ms, periods, pdts = make_workload()
    ev = 2 * N_CURVES * N_POINTS * N_PERIODS * len(PDTS)
    stream = torch.cuda.current_stream(device)
    out = {"workload": "CE(10x10) + AOV(15) + top-32 peaks, 1000 curves x 4096 points x "
                       "10000 log periods [0.1, 100] d x pdts [0, 1e-6]", "evals": ev}
    for mode, flags, k in (("chosen", nat.PF_MODE_CHOSEN, steps),
                           ("plain", nat.PF_MODE_PLAIN, 1)):
        st = BatchStep(ts, ms, periods, pdts, flags, torch, device)
        with clocks.region(f"batch_4096_{mode}"):
            ms_, _ = time_steps(st.run, k, 1, torch, flush, stream)
        out[mode] = {"ms_per_step": ms_, "value": ev / (ms_ * 1e-3)}
        st.ctx.close()
    out["chosen_over_plain"] = out["plain"]["ms_per_step"] / out["chosen"]["ms_per_step"]
    return out


# ------------------------------------------------------------------ main


def _measured_hbm_gbs():
    """The copy bandwidth measured on this pool's B200s (MEASURED_PEAKS.json
    beside this file), else the earlier measurement on the pool."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured (MEASURED_PEAKS.json)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback (earlier measurement on the pool)"


def _roofline(kernel_ms, evals_algo, pipes, off, periods, pdts):
    """Roofline of the kernel with the most time, and each kernel's
    fraction of its own bound."""
    dom = max(kernel_ms, key=kernel_ms.get)
    rf = ROOFLINE[dom]

    def frac(pipe, ops, ms):
        pk = pipes.get(pipe, {}).get("per_s", float("nan"))
        a = evals_algo * ops / (ms * 1e-3)
        return a, pk, (a / pk if pk == pk else None)

    achieved, peak, f = frac(rf["pipe"], rf["ops"], kernel_ms[dom])
    views = {}
    for name, (pipe, ops) in rf["views"].items():
        a, pk, fv = frac(pipe, ops, kernel_ms[dom])
        views[name] = {"achieved_gops": a / 1e9, "peak_gops": pk / 1e9, "ops_per_eval": ops,
                       "frac": fv}
    per_kernel = {a: {"kernel": ROOFLINE[a]["kernel"], "ms": kernel_ms[a],
                      "bound": ROOFLINE[a]["bound"],
                      "frac": frac(ROOFLINE[a]["pipe"], ROOFLINE[a]["ops"], kernel_ms[a])[2]}
                  for a in kernel_ms}
    hbm_peak, hbm_src = _measured_hbm_gbs()
    in_bytes = int(off[-1]) * 8 + len(periods) * 4
    out_bytes = (len(off) - 1) * len(periods) * len(pdts) * 4
    hbm_gbs = (in_bytes + out_bytes) / (kernel_ms[dom] * 1e-3) / 1e9
    return {"bound": rf["bound"], "kernel": rf["kernel"], "achieved": achieved / 1e9,
            "peak": peak / 1e9, "unit": "Gop/s", "frac": f, "ops_per_eval": rf["ops"],
            "kernel_ms": kernel_ms[dom],
            "peak_source": f"measured on this GPU (pipe_peaks.cu, {rf['pipe']})",
            "traffic": RAGGED_TRAFFIC[dom], "views": views, "per_kernel": per_kernel,
            "hbm_view": {"achieved_gbs": hbm_gbs, "peak_gbs": hbm_peak,
                         "frac": hbm_gbs / hbm_peak, "peak_source": hbm_src}}


def ragged_main(args):
    import torch

    from periodfind_b200 import _native as nat
    from periodfind_b200.distributed import max_over_ranks

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    # Each rank searches its own batch of curves (weak scaling, no exchange).
    n_curves = args.curves or RAGGED_CURVES
    t, m, off = lc.ragged_batch(n_curves, SEED + 5 + rank)
    periods, pdts = ragged_grid()
    evals_algo = int(off[-1]) * len(periods) * len(pdts)
    clocks = Clocks(local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    pipes = measure_pipes() if rank == 0 else {}

    step = RaggedStep(t, m, off, periods, pdts, torch, local)
    stream = step.stream
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with clocks.region("chosen"):
        ms_step, _ = time_steps(step.chosen, args.steps, args.warmup, torch, flush, stream)
    if dist:
        dist.barrier()
    ms_step = max_over_ranks(ms_step, device="cuda")
    launches = args.steps * (step.plan_kernels + 2)  # + the two preparation kernels

    with clocks.region("plain"):
        plain_ms, _ = time_steps(step.plain, max(1, min(args.steps, 3)), 1, torch, flush,
                                 stream)
    plain_ms = max_over_ranks(plain_ms, device="cuda")

    # Per algorithm: the plan's replay (CUDA events), the fold / bin kernels
    # alone (the library's events around the class launches of a direct
    # chosen call, tuned by its first call), per-curve latency.
    algo_ms, kernel_ms, latency, one_launch_ms = {}, {}, {}, {}
    for algo in ALGOS:
        plan = step.plans[algo]
        algo_ms[algo], _ = time_steps(lambda: plan.launch(stream), 3, 1, torch, flush, stream)
        step.direct(algo, nat.PF_MODE_CHOSEN, peaks=False)
        ks = []
        for _ in range(3):
            step.direct(algo, nat.PF_MODE_CHOSEN, peaks=False)
            torch.cuda.synchronize()
            ks.append(step.ctx.last_kernel_ms)
        kernel_ms[algo] = float(np.mean(ks))
        # The same kernels with every length class in one launch (one shape).
        step.direct(algo, nat.PF_MODE_CHOSEN | nat.PF_ONE_LAUNCH, peaks=False)
        torch.cuda.synchronize()
        one_launch_ms[algo] = step.ctx.last_kernel_ms
        latency[algo] = {"chosen": curve_latency(step, algo, nat.PF_MODE_CHOSEN),
                         "plain": curve_latency(step, algo, nat.PF_MODE_PLAIN)}
    step.chosen()  # the chosen peaks back in pk_i / pk_v for the precision check
    torch.cuda.synchronize()

    hb = HostBatch(t, m, off)
    with clocks.region("e2e"):
        e2e_s, h2d, d2h, e2e_launches = e2e_cabi(hb, periods, pdts, max(1, min(args.steps, 3)),
                                                 1, local)
    e2e_s = max_over_ranks(e2e_s, device="cuda")
    if dist:
        dist.barrier()

    n_eval = 3 * evals_algo * world
    if rank == 0:
        prec = ls_peak_error(step, periods, 64, torch)
        calc_s = None if args.no_calc else e2e_calc(t, m, off, periods, pdts, local)
        cpu = None if args.no_cpu else cpu_baseline(t, m, off, periods, pdts)
        ref_cuda = None if args.no_cpu else reference_cuda(t, m, off, periods, pdts, clocks)
        secondary = batch_secondary(torch, local, flush, clocks)
        lens = np.diff(off)
        line = {
            "metric": METRIC, "value": n_eval / (ms_step * 1e-3), "unit": "evals/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 bin fold (CE, AOV), split-precision f32 phase (LS), f32 / "
                     "fixed-point statistics",
            "data": "synthetic",
            "config": {"workload": RAGGED_WORKLOAD, "curves_per_gpu": n_curves,
                       "points_per_gpu": int(off[-1]), "mean_length": float(lens.mean()),
                       "periods": len(periods), "pdts": [0.0], "evals_per_step": n_eval,
                       "l2": "inputs (326 MB) and periodogram (8 GB) larger than L2; L2 also "
                             "flushed (256 MB write) between timed steps",
                       "parallelism": f"{world} independent replicas (curves sharded)"},
            "plain": {"value": n_eval / (plain_ms * 1e-3), "ms_per_step": plain_ms,
                      "chosen_over_plain": plain_ms / ms_step},
            "chosen_over_plain": plain_ms / ms_step,
            "e2e": {"value": n_eval / e2e_s, "unit": "evals/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3,
                    "path": "C ABI pf_ce_peaks / pf_aov_peaks / pf_ls_peaks from per-curve host "
                            "arrays (PF_ASYNC pipeline, CE in two calls), magnitude preparation "
                            "fused into the packing (PF_HOST_NORMALIZE / PF_HOST_CENTER) "
                            "inside the step"},
            "e2e_calc": None if calc_s is None else {
                "s_per_algo": calc_s, "value": n_eval / sum(calc_s.values()),
                "path": "gpu.ConditionalEntropy / AOV / LombScargle .calc(list of numpy, "
                        "output='peaks'), 3.2e6 Statistics objects per algorithm"},
            "algo_ms": algo_ms, "kernels_ms": kernel_ms,
            "kernels_ms_one_launch": one_launch_ms,
            "tuning": step.ctx.tuning_report().strip().splitlines(),
            "latency_per_curve": latency,
            "ls_peak_frequency_error": prec,
            "roofline": _roofline(kernel_ms, evals_algo, pipes, off, periods, pdts),
            "pipes": {k: round(v["per_s"] / 1e12, 3) for k, v in pipes.items()},
            "cpu_baseline": cpu,
            "reference_cuda": ref_cuda,
            "batch_4096": secondary,
            "clocks": clocks.regions["chosen"],
            "clocks_regions": clocks.regions,
            "gpu_launches": int(launches),
            "e2e_gpu_launches_per_step": e2e_launches,
        }
        print(json.dumps(line), flush=True)
    step.close()
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--curves", type=int, default=0,
                    help="curves per GPU (default: the workload's own count)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU and reference baselines")
    ap.add_argument("--no-calc", action="store_true", help="skip the Python calc() path")
    ap.add_argument("--workload", default="ragged",
                    choices=["ragged", "batch", "small", "lsgrad", "precision", "fpw", "bls",
                             "device", "profile", "profile_batch"],
                    help="'ragged' (default): the mixed ragged batch; separate reports on 1 "
                         "GPU: 'batch' CE + AOV on 1000 x 4096, 'small' CE stats on 100 x "
                         "1024, 'lsgrad' LS derivatives and Newton refinement, 'precision' LS "
                         "folds on the precision-study batch, 'fpw' / 'bls' on the 1000 x 4096 "
                         "batch, 'device' device-resident periodograms, 'profile' / "
                         "'profile_batch' short runs for ncu captures")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.workload == "ragged":
        ragged_main(args)
        return
    from bench_reports import ARMS

    ARMS[args.workload](args)


if __name__ == "__main__":
    main()
