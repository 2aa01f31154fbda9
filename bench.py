"""Benchmark: curve x period x point evaluations per second on B200.

Workload (one "step"): Conditional Entropy (10 x 10 bins) and AOV (15 bins)
periodograms plus the top-32 peak search, over 1000 light curves x 4096
points, 10000 trial periods log-spaced in [0.1, 100] days and period
derivatives [0, 1e-6] -- 2 x 8.19e10 evaluations per step.  Synthetic
curves (seeded): half sinusoids, a quarter sawtooth, a quarter box eclipses
(depth 0.5, duty 0.05) with N(0, 0.05^2) noise, times uniform over 2000 days.

Reported (one JSON line on rank 0):
  value     evals/s of the chosen form, inputs resident in HBM, device-timed
            with CUDA events around each step (max over ranks); L2 is
            flushed (256 MB write) between timed steps, outside the events.
  e2e       the same metric through the public API (gpu.ConditionalEntropy /
            gpu.AOV .calc(..., output='peaks')) with host numpy inputs: the
            timed region includes magnitude preparation, the H2D copy of the
            step's inputs and the D2H copy of the peaks.
  plain     the plain form (the reference's fold, op for op) on the same
            device-resident workload, for the chosen-vs-plain ratio.
  roofline  the dominant fold kernel against the measured FP64-pipe peak
            (this path is FP64/XU issue bound; HBM traffic is given too).
  cpu_baseline  the oracle (C/OpenMP restatement of the reference's Rust
            CPU path) on all host cores over a bounded sample of curves.

--impl reference runs that CPU restatement (the reference's CPU
implementation is Rust; no Rust toolchain exists on these machines) as the
reference arm, on rank 0 only.
"""

from __future__ import annotations

import argparse
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

N_CURVES = 1000
N_POINTS = 4096
N_PERIODS = 10000
PDTS = (0.0, 1e-6)
N_PEAKS = 32
SEED = 20261205
WORKLOAD = "CE(10x10)+AOV(15)+top32 peaks, 1000 curves x 4096 pts, 10000 log periods [0.1,100] d x pdts [0,1e-6]"
METRIC = "curve*period*point evals/s on 1 B200, chosen vs plain, at stated error"


def make_workload(n_curves=N_CURVES, seed=SEED):
    from tests import lightcurves as lc

    ts, ms = lc.mixed_signal_batch(n_curves, N_POINTS, seed)
    periods = np.exp(np.linspace(np.log(0.1), np.log(100.0), N_PERIODS)).astype(np.float32)
    pdts = np.array(PDTS, np.float32)
    return ts, ms, periods, pdts


def evals_per_step(n_curves):
    return 2 * n_curves * N_POINTS * N_PERIODS * len(PDTS)


# ----------------------------------------------------------------- clocks


class ClockSampler:
    """nvidia-smi samples (200 ms) while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

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
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        mhz, mx, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                mx = float(parts[2])
                power.append(float(parts[3]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz),
                "power_w_max": max(power) if power else None}


# -------------------------------------------------------------- pipe peaks


def measure_pipes():
    import ctypes

    lib = ctypes.CDLL(os.path.join(ROOT, "periodfind_b200", "libpfpeaks.so"))

    class R(ctypes.Structure):
        _fields_ = [("name", ctypes.c_char * 32), ("ops_per_clk_per_sm", ctypes.c_double),
                    ("ops_per_s", ctypes.c_double), ("sm_mhz", ctypes.c_double)]

    arr = (R * 32)()
    k = lib.pfpk_measure(0, arr, 32)
    return {arr[i].name.decode(): {"per_s": arr[i].ops_per_s,
                                   "per_clk_sm": arr[i].ops_per_clk_per_sm,
                                   "mhz": arr[i].sm_mhz} for i in range(max(k, 0))}


# ----------------------------------------------------------- device step


class DeviceStep:
    """CE + AOV + peaks on device-resident packed curves via the C ABI."""

    def __init__(self, ts, ms, periods, pdts, mode_flags, torch, device=0):
        from periodfind_b200 import _native as nat
        from tests import lightcurves as lc

        self.nat = nat
        self.torch = torch
        self.ctx = nat.default_context(device)
        self.flags = mode_flags
        off = np.zeros(len(ts) + 1, np.int64)
        np.cumsum([len(t) for t in ts], out=off[1:])
        self.off = off
        dev = "cuda"
        self.t = torch.from_numpy(np.concatenate(ts)).to(dev)
        self.m_ce = torch.from_numpy(np.concatenate([lc.normalize(m) for m in ms])).to(dev)
        self.m_aov = torch.from_numpy(np.concatenate(ms)).to(dev)
        self.P = torch.from_numpy(periods).to(dev)
        self.D = torch.from_numpy(pdts).to(dev)
        n = len(ts)
        self.n = n
        cells = len(periods) * len(pdts)
        self.cells = cells
        self.pg_ce = torch.empty((n, cells), dtype=torch.float32, device=dev)
        self.pg_aov = torch.empty((n, cells), dtype=torch.float32, device=dev)
        self.pk_idx = torch.empty((2, n, N_PEAKS), dtype=torch.int64, device=dev)
        self.pk_val = torch.empty((2, n, N_PEAKS), dtype=torch.float32, device=dev)
        self.np_ = len(periods)
        self.nd = len(pdts)

    def run(self, stream):
        c, lib, h, nat = self.ctx, self.ctx.lib, self.ctx.handle, self.nat
        c.check(lib.pf_ce_dev(h, self.t.data_ptr(), self.m_ce.data_ptr(), self.off.ctypes.data,
                              self.n, self.P.data_ptr(), self.np_, self.D.data_ptr(), self.nd,
                              10, 10, 1, 1, self.flags, self.pg_ce.data_ptr(), stream))
        c.check(lib.pf_find_peaks_dev(h, self.pg_ce.data_ptr(), self.n, self.cells, N_PEAKS, 1,
                                      0, self.pk_idx[0].data_ptr(), self.pk_val[0].data_ptr(),
                                      stream))
        c.check(lib.pf_aov_dev(h, self.t.data_ptr(), self.m_aov.data_ptr(), self.off.ctypes.data,
                               self.n, self.P.data_ptr(), self.np_, self.D.data_ptr(), self.nd,
                               15, 1, self.flags, self.pg_aov.data_ptr(), stream))
        c.check(lib.pf_find_peaks_dev(h, self.pg_aov.data_ptr(), self.n, self.cells, N_PEAKS, 1,
                                      1, self.pk_idx[1].data_ptr(), self.pk_val[1].data_ptr(),
                                      stream))


def time_device(step, steps, warmup, torch, flush):
    stream = torch.cuda.current_stream()
    s = stream.cuda_stream
    for _ in range(warmup):
        step.run(s)
    torch.cuda.synchronize()
    launches0 = step.ctx.launches
    total = 0.0
    for _ in range(steps):
        flush.zero_()  # evict L2 between timed steps (outside the events)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step.run(s)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    return total / steps, step.ctx.launches - launches0


def time_kernels(step, torch, reps=3):
    """Average duration of the CE and AOV fold kernels (their own events)."""
    s = torch.cuda.current_stream().cuda_stream
    ce, aov = [], []
    c, lib, h = step.ctx, step.ctx.lib, step.ctx.handle
    for _ in range(reps):
        c.check(lib.pf_ce_dev(h, step.t.data_ptr(), step.m_ce.data_ptr(), step.off.ctypes.data,
                              step.n, step.P.data_ptr(), step.np_, step.D.data_ptr(), step.nd,
                              10, 10, 1, 1, step.flags, step.pg_ce.data_ptr(), s))
        torch.cuda.synchronize()
        ce.append(c.last_kernel_ms)
        c.check(lib.pf_aov_dev(h, step.t.data_ptr(), step.m_aov.data_ptr(), step.off.ctypes.data,
                               step.n, step.P.data_ptr(), step.np_, step.D.data_ptr(), step.nd,
                               15, 1, step.flags, step.pg_aov.data_ptr(), s))
        torch.cuda.synchronize()
        aov.append(c.last_kernel_ms)
    return float(np.mean(ce)), float(np.mean(aov))


def time_e2e(ts, ms, periods, pdts, steps, warmup, device=0):
    from periodfind_b200 import gpu

    ce = gpu.ConditionalEntropy(10, 10, device=device)
    aov = gpu.AOV(15, device=device)
    for _ in range(warmup):
        ce.calc(ts, ms, periods, pdts, output="peaks", n_peaks=N_PEAKS)
        aov.calc(ts, ms, periods, pdts, output="peaks", n_peaks=N_PEAKS)
    t0 = time.perf_counter()
    for _ in range(steps):
        a = ce.calc(ts, ms, periods, pdts, output="peaks", n_peaks=N_PEAKS)
        b = aov.calc(ts, ms, periods, pdts, output="peaks", n_peaks=N_PEAKS)
    dt = (time.perf_counter() - t0) / steps
    assert len(a) == len(ts) and len(b) == len(ts)
    return dt


# ------------------------------------------------------------ CPU baseline


def cpu_baseline(ts, ms, periods, pdts, target_s=12.0):
    """The oracle (C/OpenMP restatement of the reference's Rust path) on all
    host cores over the first k curves, k sized for ~target_s of work."""
    from oracle import oracle as O
    from tests import lightcurves as lc

    cores = os.cpu_count() or 1
    k = 1
    t0 = time.perf_counter()
    O.ce(ts[:k], [lc.normalize(m) for m in ms[:k]], periods, pdts, 10, 10, n_threads=cores)
    O.aov(ts[:k], ms[:k], periods, pdts, 15, n_threads=cores)
    one = time.perf_counter() - t0
    k = int(max(1, min(len(ts), target_s / max(one, 1e-3))))
    t0 = time.perf_counter()
    O.ce(ts[:k], [lc.normalize(m) for m in ms[:k]], periods, pdts, 10, 10, n_threads=cores)
    O.aov(ts[:k], ms[:k], periods, pdts, 15, n_threads=cores)
    dt = time.perf_counter() - t0
    value = evals_per_step(k) / dt
    return {"value": value, "unit": "evals/s", "cores": cores, "kind": "port",
            "sample": f"{k} of {len(ts)} curves (CE 10x10 + AOV 15, full 10000x2 grid), "
                      f"{dt:.1f} s on {cores} threads"}


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ts, ms, periods, pdts = make_workload()
    from oracle import oracle as O
    from tests import lightcurves as lc

    cores = os.cpu_count() or 1
    k = 2
    sub_t, sub_m = ts[:k], ms[:k]
    run = lambda: (O.ce(sub_t, [lc.normalize(m) for m in sub_m], periods, pdts, 10, 10,
                        n_threads=cores),
                   O.aov(sub_t, sub_m, periods, pdts, 15, n_threads=cores))
    for _ in range(args.warmup):
        run()
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        run()
        times.append(time.perf_counter() - t0)
    per_step = float(np.mean(times))
    value = evals_per_step(k) / per_step
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "evals/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": per_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 fold, f32 statistics", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_curves_per_step": k},
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": cores, "kind": "port",
                         "sample": f"{k} of {N_CURVES} curves per step, full grid, "
                                   f"C/OpenMP restatement of the reference's Rust CPU path"},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------ ragged batch


def make_ragged(n_curves=100000, seed=SEED + 5, n_periods=20000):
    """Mixed ragged batch: lengths lognormal (median 300, sigma 0.8) clipped to
    [20, 2000]; seasonal cadence over 2500 days (125-day seasons); 1/3
    sinusoids, 1/3 box eclipses (depth 0.5, duty 0.05), 1/3 pure noise; noise
    sigma U[0.02, 0.1]; 20000 periods log-spaced in [0.05, 500] days."""
    rng = np.random.default_rng(seed)
    lens = np.clip(np.round(rng.lognormal(np.log(300.0), 0.8, n_curves)), 20, 2000).astype(np.int64)
    cid = np.repeat(np.arange(n_curves), lens)
    n_years = int(np.ceil(2500.0 / 365.25))
    t = rng.integers(0, n_years, cid.size) * 365.25 + rng.uniform(0.0, 125.25, cid.size)
    t = np.minimum(t, 2500.0)
    order = np.lexsort((t, cid))
    t = t[order].astype(np.float32)
    period = np.exp(rng.uniform(np.log(0.05), np.log(500.0), n_curves))[cid]
    phase = rng.uniform(0, 1, n_curves)[cid]
    kind = (np.arange(n_curves) % 3)[cid]
    sigma = rng.uniform(0.02, 0.1, n_curves)[cid]
    ph = np.mod(t / period + phase, 1.0)
    y = np.where(kind == 0, 0.3 * np.sin(2 * np.pi * ph),
                 np.where(kind == 1, np.where(ph < 0.05, -0.5, 0.0), 0.0))
    m = (15.0 + y + rng.normal(0.0, 1.0, cid.size) * sigma).astype(np.float32)
    off = np.zeros(n_curves + 1, np.int64)
    np.cumsum(lens, out=off[1:])
    periods = np.exp(np.linspace(np.log(0.05), np.log(500.0), n_periods)).astype(np.float32)
    return t, m, off, periods, np.zeros(1, np.float32)


def ragged_arm(args):
    import torch

    from periodfind_b200 import _native as nat

    torch.cuda.set_device(0)
    n_curves = args.curves if args.curves != N_CURVES else 100000
    t, m, off, periods, pdts = make_ragged(n_curves)
    lens = np.diff(off)
    ctx = nat.default_context(0)
    dev = "cuda"
    d_t = torch.from_numpy(t).to(dev)
    # Per-curve magnitude preparation as the reference does it: normalise for
    # CE (periodfind/_utils.py:39-45), centre for LS, raw for AOV.
    seg_min = np.minimum.reduceat(m, off[:-1])
    seg_max = np.maximum.reduceat(m, off[:-1])
    cid = np.repeat(np.arange(n_curves), lens)
    m_ce = (((m - seg_min[cid]) / (seg_max[cid] - seg_min[cid])) * np.float32(0.999)
            + np.float32(5e-4)).astype(np.float32)
    seg_mean = (np.add.reduceat(m.astype(np.float64), off[:-1]) / lens).astype(np.float32)
    m_ls = (m - seg_mean[cid]).astype(np.float32)
    mags = {"ce": torch.from_numpy(m_ce).to(dev), "aov": torch.from_numpy(m).to(dev),
            "ls": torch.from_numpy(m_ls).to(dev)}
    d_p = torch.from_numpy(periods).to(dev)
    d_d = torch.from_numpy(pdts).to(dev)
    cells = len(periods) * len(pdts)
    pg = torch.empty((n_curves, cells), dtype=torch.float32, device=dev)
    pk_i = torch.empty((n_curves, N_PEAKS), dtype=torch.int64, device=dev)
    pk_v = torch.empty((n_curves, N_PEAKS), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream()
    s = stream.cuda_stream
    evals = int(lens.sum()) * cells

    def step(algo, flags):
        h, lib = ctx.handle, ctx.lib
        common = (h, d_t.data_ptr(), mags[algo].data_ptr(), off.ctypes.data, n_curves,
                  d_p.data_ptr(), len(periods), d_d.data_ptr(), len(pdts))
        if algo == "ce":
            ctx.check(lib.pf_ce_dev(*common, 10, 10, 1, 1, flags, pg.data_ptr(), s))
        elif algo == "aov":
            ctx.check(lib.pf_aov_dev(*common, 15, 1, flags, pg.data_ptr(), s))
        else:
            ctx.check(lib.pf_ls_dev(*common, flags, pg.data_ptr(), s))
        ctx.check(lib.pf_find_peaks_dev(h, pg.data_ptr(), n_curves, cells, N_PEAKS, 1,
                                        0 if algo == "ce" else 1, pk_i.data_ptr(),
                                        pk_v.data_ptr(), s))

    out = {"workload": f"ragged: {n_curves} curves, lengths lognormal(median 300, sigma 0.8) "
                       f"in [20, 2000] (mean {lens.mean():.0f}), seasonal cadence 2500 d, "
                       f"{len(periods)} log periods [0.05, 500] d, top-{N_PEAKS} peaks",
           "evals_per_algo": evals, "algos": {}}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    from periodfind_b200.plan import BatchPlan

    for algo in ("ce", "aov", "ls"):
        row = {}
        # The chosen form runs as a batch plan: the pipeline (packing,
        # preparation, per-length-class tuned queue launches, peaks) captured
        # once as a CUDA graph; the plain form as direct calls per step.
        plan = BatchPlan(algo, d_t, mags[algo], off, d_p, d_d, pg, n_phase=10 if algo == "ce"
                         else 15, n_mag=10, flags=nat.PF_MODE_CHOSEN, n_peaks=N_PEAKS,
                         peak_idx=pk_i, peak_val=pk_v)
        for mode, flags in (("chosen", nat.PF_MODE_CHOSEN), ("plain", nat.PF_MODE_PLAIN)):
            run = (lambda: plan.launch(stream)) if mode == "chosen" else (
                lambda flags=flags: step(algo, flags))
            run()
            torch.cuda.synchronize()
            ts_ = []
            for _ in range(max(1, args.steps)):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                run()
                e1.record(stream)
                e1.synchronize()
                ts_.append(e0.elapsed_time(e1))
            ms_ = float(np.median(ts_))
            # Per-curve device latency from a separate, stamped run.
            step(algo, flags | nat.PF_TIMING)
            lat = np.zeros(n_curves)
            ctx.check(ctx.lib.pf_curve_latency(ctx.handle, n_curves, lat.ctypes.data))
            row[mode] = {"ms": ms_, "evals_per_s": evals / (ms_ * 1e-3),
                         "curve_latency_ms_p50": float(np.percentile(lat, 50)) / 1e6,
                         "curve_latency_ms_p99": float(np.percentile(lat, 99)) / 1e6}
        row["chosen_over_plain"] = row["plain"]["ms"] / row["chosen"]["ms"]
        row["chosen"]["launch"] = "batch plan (CUDA graph replay)"
        plan.close()
        out["algos"][algo] = row
    tc = sum(out["algos"][a]["chosen"]["ms"] for a in out["algos"])
    tp = sum(out["algos"][a]["plain"]["ms"] for a in out["algos"])
    out["all_three"] = {"chosen_evals_per_s": 3 * evals / (tc * 1e-3),
                        "plain_evals_per_s": 3 * evals / (tp * 1e-3),
                        "chosen_over_plain": tp / tc}
    out["tuning"] = ctx.tuning_report().strip().splitlines()
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ FPW


def fpw_arm(args, bls=False):
    """FPW(10) -- or, with bls, BoxLeastSquares(50, 0.01, 0.5) -- over the
    benchmark batch (1000 curves x 4096 points, 10000 log periods in
    [0.1, 100] d x pdts [0, 1e-6]) with per-point uncertainties U[0.02, 0.1]:
    device time of the chosen and plain forms (the kernel, CUDA events),
    end-to-end calc(output='peaks') from numpy lists, and the oracle (the
    Rust path's restatement) on all host cores over a sample."""
    from periodfind_b200 import gpu

    ts, ms, periods, pdts = make_workload(args.curves)
    rng = np.random.default_rng(SEED + 6)
    es = [rng.uniform(0.02, 0.1, len(t)).astype(np.float32) for t in ts]
    evals = sum(len(t) for t in ts) * len(periods) * len(pdts)
    label = "BLS(50, qmin 0.01, qmax 0.5)" if bls else "FPW(10)"
    out = {"workload": f"{label}, {len(ts)} curves x {N_POINTS} pts, {N_PERIODS} log periods "
                       f"[0.1,100] d x pdts {list(PDTS)}, errs U[0.02,0.1]", "evals": evals}
    from periodfind_b200 import _native as nat

    ctx = nat.default_context(0)
    for mode in ("chosen", "plain"):
        obj = gpu.BoxLeastSquares(50, 0.01, 0.5, mode=mode) if bls else gpu.FPW(10, mode=mode)
        obj.periodograms(ts, ms, periods, pdts, errs=es)
        k = []
        for _ in range(max(1, args.steps)):
            obj.periodograms(ts, ms, periods, pdts, errs=es)
            k.append(ctx.lib.pf_last_kernel_ms(ctx.handle))
        kms = float(np.median(k))
        obj.calc(ts, ms, periods, pdts, errs=es, output="peaks", n_peaks=N_PEAKS)
        w = []
        for _ in range(max(1, min(args.steps, 3))):
            t0 = time.perf_counter()
            obj.calc(ts, ms, periods, pdts, errs=es, output="peaks", n_peaks=N_PEAKS)
            w.append(time.perf_counter() - t0)
        out[mode] = {"kernel_ms": kms, "evals_per_s": evals / (kms * 1e-3),
                     "e2e_ms": float(np.median(w)) * 1e3,
                     "e2e_evals_per_s": evals / float(np.median(w))}
    out["chosen_over_plain"] = out["plain"]["kernel_ms"] / out["chosen"]["kernel_ms"]
    if not args.no_cpu:
        from oracle import oracle as O

        cores = os.cpu_count() or 1
        k = 20
        t0 = time.perf_counter()
        if bls:
            O.bls(ts[:k], ms[:k], periods, pdts, 50, 0.01, 0.5, errs=es[:k], n_threads=cores)
        else:
            O.fpw(ts[:k], ms[:k], periods, pdts, 10, errs=es[:k], n_threads=cores)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": k * N_POINTS * N_PERIODS * len(PDTS) / dt,
                               "unit": "evals/s", "cores": cores, "kind": "port",
                               "sample": f"{k} of {len(ts)} curves, {dt:.1f} s"}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------- device-resident I/O


def device_arm(args):
    """CE(10x10) and AOV(15) periodograms of the benchmark batch (1000 curves x
    4096 points x 10000 periods x 2 pdts) from curves already on the GPU,
    left on the GPU (periodograms_device: magnitude preparation on the
    device, no host copy), against the public host path
    calc(output='periodogram') from numpy lists, which returns the 80 MB
    periodogram per algorithm to the host.  Wall time per step, synchronised."""
    import torch

    from periodfind_b200 import gpu

    torch.cuda.set_device(0)
    ts, ms, periods, pdts = make_workload(args.curves)
    off = np.zeros(len(ts) + 1, np.int64)
    np.cumsum([len(t) for t in ts], out=off[1:])
    d_t = torch.from_numpy(np.concatenate(ts)).cuda()
    d_m = torch.from_numpy(np.concatenate(ms)).cuda()
    evals = 2 * int(off[-1]) * len(periods) * len(pdts)
    ce, aov = gpu.ConditionalEntropy(10, 10), gpu.AOV(15)

    def dev_step():
        a = ce.periodograms_device(d_t, d_m, off, periods, pdts)
        b = aov.periodograms_device(d_t, d_m, off, periods, pdts)
        torch.cuda.synchronize()
        return a, b

    def host_step():
        return (ce.calc(ts, ms, periods, pdts, output="periodogram"),
                aov.calc(ts, ms, periods, pdts, output="periodogram"))

    out = {"workload": f"CE(10x10) + AOV(15) periodograms, {len(ts)} curves x {N_POINTS} pts x "
                       f"{N_PERIODS} periods x {len(PDTS)} pdts", "evals": evals}
    for name, fn in (("device_resident", dev_step), ("host_calc_periodogram", host_step)):
        for _ in range(2):
            fn()
        w = []
        for _ in range(max(3, args.steps)):
            t0 = time.perf_counter()
            fn()
            w.append(time.perf_counter() - t0)
        ms_ = float(np.median(w)) * 1e3
        out[name] = {"ms": ms_, "evals_per_s": evals / (ms_ * 1e-3)}
    print(json.dumps(out), flush=True)


# ------------------------------------------------------ small CE batch


def small_arm(args):
    """CE 10 x 10 on 100 curves x 1024 points (times uniform in [0, 1000] d,
    15 + 0.3 sin(2 pi t / P + phi) + N(0, 0.05^2), P ~ U[0.5, 10] d) over
    1000 periods linspace(0.5, 10) d, period_dts [0], output 'stats'.
    Device time of the chosen and plain forms, end-to-end calc() time, bin
    agreement of the two forms, and the CPU port on all host cores."""
    import torch

    from periodfind_b200 import _native as nat
    from periodfind_b200 import gpu

    torch.cuda.set_device(0)
    rng = np.random.default_rng(SEED + 1)
    n_curves, n_pts = 100, 1024
    ts, ms = [], []
    for _ in range(n_curves):
        t = np.sort(rng.uniform(0.0, 1000.0, n_pts)).astype(np.float32)
        per, ph = rng.uniform(0.5, 10.0), rng.uniform(0.0, 2 * np.pi)
        m = 15.0 + 0.3 * np.sin(2 * np.pi * t.astype(np.float64) / per + ph)
        ts.append(t)
        ms.append((m + rng.normal(0.0, 0.05, n_pts)).astype(np.float32))
    periods = np.linspace(0.5, 10.0, 1000).astype(np.float32)
    pdts = np.zeros(1, np.float32)
    evals = n_curves * n_pts * len(periods)
    msn = [((m - m.min()) / (m.max() - m.min()) * np.float32(0.999) + np.float32(5e-4))
           .astype(np.float32) for m in ms]
    off = np.arange(n_curves + 1, dtype=np.int64) * n_pts
    d_t = torch.from_numpy(np.concatenate(ts)).cuda()
    d_m = torch.from_numpy(np.concatenate(msn)).cuda()
    d_p = torch.from_numpy(periods).cuda()
    d_d = torch.from_numpy(pdts).cuda()
    pg = torch.empty((n_curves, len(periods)), device="cuda")
    ctx = nat.default_context(0)
    s = torch.cuda.current_stream().cuda_stream
    out = {"workload": "CE 10x10 stats, 100 curves x 1024 points x 1000 periods "
                       "linspace(0.5, 10) d, period_dts [0]", "evals": evals}
    for mode, flags in (("chosen", nat.PF_MODE_CHOSEN), ("plain", nat.PF_MODE_PLAIN)):
        def run(flags=flags):
            ctx.check(ctx.lib.pf_ce_dev(ctx.handle, d_t.data_ptr(), d_m.data_ptr(),
                                        off.ctypes.data, n_curves, d_p.data_ptr(), len(periods),
                                        d_d.data_ptr(), 1, 10, 10, 1, 1, flags, pg.data_ptr(), s))
        for _ in range(3):
            run()
        torch.cuda.synchronize()
        k = []
        for _ in range(max(3, args.steps)):
            run()
            torch.cuda.synchronize()
            k.append(ctx.lib.pf_last_kernel_ms(ctx.handle))
        obj = gpu.ConditionalEntropy(10, 10, mode=mode)
        obj.calc(ts, ms, periods, pdts, output="stats")
        w = []
        for _ in range(max(3, args.steps)):
            t0 = time.perf_counter()
            obj.calc(ts, ms, periods, pdts, output="stats")
            w.append(time.perf_counter() - t0)
        kms, ws = float(np.median(k)), float(np.median(w))
        out[mode] = {"kernel_ms": kms, "evals_per_s": evals / (kms * 1e-3),
                     "e2e_ms": ws * 1e3, "e2e_evals_per_s": evals / ws}
    a = gpu.ConditionalEntropy(mode="plain").periodograms(ts, msn, periods, pdts)
    b = gpu.ConditionalEntropy(mode="chosen", reference_stats=True).periodograms(
        ts, msn, periods, pdts)
    out["bins_identical_chosen_vs_plain"] = bool(np.array_equal(a, b))
    out["chosen_over_plain"] = out["plain"]["kernel_ms"] / out["chosen"]["kernel_ms"]
    if not args.no_cpu:
        from oracle import oracle as O

        cores = os.cpu_count() or 1
        t0 = time.perf_counter()
        O.ce(ts, msn, periods, pdts, 10, 10, n_threads=cores)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": evals / dt, "unit": "evals/s", "cores": cores,
                               "kind": "port", "sample": f"all {n_curves} curves, {dt:.2f} s"}
    print(json.dumps(out), flush=True)


# ------------------------------------------------- LS derivatives and study


def _seasonal_ls_batch(lengths, seed, baseline=3000.0):
    """LS study curves: seasonal cadence over `baseline` days (240-day annual
    gap), 15 + A sin(2 pi f t) + N(0, sigma^2) with A ~ U[0.01, 0.5],
    sigma ~ U[0.01, 0.1], f ~ U[0.01, 20] / day; magnitudes centred.
    Returns CSR (times, mags, offsets)."""
    rng = np.random.default_rng(seed)
    lengths = np.asarray(lengths, np.int64)
    n_curves = len(lengths)
    cid = np.repeat(np.arange(n_curves), lengths)
    n_years = int(np.ceil(baseline / 365.25))
    t = rng.integers(0, n_years, cid.size) * 365.25 + rng.uniform(0.0, 125.25, cid.size)
    t = np.minimum(t, baseline)
    t = t[np.lexsort((t, cid))].astype(np.float32)
    amp = rng.uniform(0.01, 0.5, n_curves)[cid]
    sig = rng.uniform(0.01, 0.1, n_curves)[cid]
    f = rng.uniform(0.01, 20.0, n_curves)[cid]
    ph = rng.uniform(0, 2 * np.pi, n_curves)[cid]
    m = 15.0 + amp * np.sin(2 * np.pi * f * t.astype(np.float64) + ph)
    m = m + rng.normal(0.0, 1.0, cid.size) * sig
    off = np.zeros(n_curves + 1, np.int64)
    np.cumsum(lengths, out=off[1:])
    mean = np.add.reduceat(m, off[:-1]) / lengths
    return t, (m - mean[cid]).astype(np.float32), off


def _event_ms(torch, fn, reps, flush):
    ts_ = []
    for _ in range(reps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        e1.synchronize()
        ts_.append(e0.elapsed_time(e1))
    return float(np.median(ts_))


def lsgrad_arm(args):
    """2000 curves x 2048 points over 3000 days; 20000 log-spaced frequencies
    in [0.01, 20] / day.  Times the LS grid periodogram + top-32 peaks, the
    autograd forward (power, dP/domega, coefficients) and backward
    (dP/dy and dL/domega) over the grid, and 5 Newton steps on the top-32
    peaks of every curve."""
    import torch

    from periodfind_b200 import _native as nat
    from periodfind_b200 import ls_grad

    torch.cuda.set_device(0)
    n_curves, n_pts, n_freq = 2000, 2048, 20000
    t, m, off = _seasonal_ls_batch(np.full(n_curves, n_pts), SEED + 4)
    freqs = np.exp(np.linspace(np.log(0.01), np.log(20.0), n_freq))
    periods = (1.0 / freqs[::-1]).astype(np.float32)
    dev = "cuda"
    d_t, d_m = torch.from_numpy(t).to(dev), torch.from_numpy(m).to(dev)
    d_p = torch.from_numpy(periods).to(dev)
    d_d = torch.zeros(1, dtype=torch.float32, device=dev)
    pg = torch.empty((n_curves, n_freq), dtype=torch.float32, device=dev)
    pk_i = torch.empty((n_curves, N_PEAKS), dtype=torch.int64, device=dev)
    pk_v = torch.empty((n_curves, N_PEAKS), dtype=torch.float32, device=dev)
    ctx = nat.default_context(0)
    s = torch.cuda.current_stream().cuda_stream
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    reps = max(1, args.steps)

    def grid_peaks():
        ctx.check(ctx.lib.pf_ls_dev(ctx.handle, d_t.data_ptr(), d_m.data_ptr(), off.ctypes.data,
                                    n_curves, d_p.data_ptr(), n_freq, d_d.data_ptr(), 1,
                                    nat.PF_MODE_CHOSEN, pg.data_ptr(), s))
        ctx.check(ctx.lib.pf_find_peaks_dev(ctx.handle, pg.data_ptr(), n_curves, n_freq, N_PEAKS,
                                            1, 1, pk_i.data_ptr(), pk_v.data_ptr(), s))

    w_grid = torch.from_numpy(2 * np.pi / periods.astype(np.float64)).to(dev)
    y = d_m.clone().requires_grad_(True)
    w = w_grid.clone().requires_grad_(True)
    holder = {}

    def forward():
        holder["P"] = ls_grad.ls_power(d_t, y, w, off)

    def backward():
        holder["P"].backward(holder["g"])

    grid_peaks()
    forward()
    holder["g"] = torch.ones_like(holder["P"])
    backward()
    torch.cuda.synchronize()
    out = {"workload": f"LS derivatives: {n_curves} curves x {n_pts} points, seasonal cadence "
                       f"3000 d, {n_freq} log-spaced frequencies [0.01, 20] / d, top-{N_PEAKS} "
                       "peaks refined by 5 Newton steps"}
    ev = n_curves * n_pts * n_freq
    ms_grid = _event_ms(torch, grid_peaks, reps, flush)
    ms_fwd = _event_ms(torch, forward, reps, flush)
    ms_bwd = []
    for _ in range(reps):
        forward()
        torch.cuda.synchronize()
        ms_bwd.append(_event_ms(torch, backward, 1, flush))
    ms_bwd = float(np.median(ms_bwd))
    # Newton refinement of the grid peaks.
    idx = pk_i.clamp(min=0)
    wg = w_grid
    w0 = wg[idx]
    hw = torch.maximum((wg[(idx - 1).clamp(min=0)] - w0).abs(),
                       (wg[(idx + 1).clamp(max=n_freq - 1)] - w0).abs()).contiguous()
    w0 = w0.contiguous()

    def refine():
        holder["ref"] = ls_grad.refine_peaks(d_t, d_m, w0, hw, off, n_steps=5)

    refine()
    ms_ref = _event_ms(torch, refine, reps, flush)
    ev_ref = n_curves * n_pts * N_PEAKS * 6
    out["grid_periodogram_peaks"] = {"ms": ms_grid, "evals_per_s": ev / (ms_grid * 1e-3)}
    out["autograd_forward"] = {"ms": ms_fwd, "evals_per_s": ev / (ms_fwd * 1e-3)}
    out["autograd_backward"] = {"ms": ms_bwd, "evals_per_s": ev / (ms_bwd * 1e-3)}
    out["newton_refine_5_steps"] = {"ms": ms_ref, "evals_per_s": ev_ref / (ms_ref * 1e-3),
                                    "peaks": n_curves * N_PEAKS}
    print(json.dumps(out), flush=True)


def precision_arm(args):
    """10000 curves, lengths log-uniform in [64, 16384], seasonal cadence over
    3000 days; 50000 frequencies uniform in [0.01, 20] / day.  Times the LS
    periodogram with each fold: plain (the reference's FP64-divide fold),
    chosen split-precision, chosen exact, and the all-FP32 fold."""
    import torch

    from periodfind_b200 import _native as nat

    torch.cuda.set_device(0)
    rng = np.random.default_rng(SEED + 3)
    n_curves = args.curves if args.curves != N_CURVES else 10000
    lengths = np.exp(rng.uniform(np.log(64), np.log(16384), n_curves)).astype(np.int64)
    t, m, off = _seasonal_ls_batch(lengths, SEED + 3)
    n_freq = 50000
    periods = (1.0 / np.linspace(0.01, 20.0, n_freq)[::-1]).astype(np.float32)
    dev = "cuda"
    d_t, d_m = torch.from_numpy(t).to(dev), torch.from_numpy(m).to(dev)
    d_p = torch.from_numpy(periods).to(dev)
    d_d = torch.zeros(1, dtype=torch.float32, device=dev)
    pg = torch.empty((n_curves, n_freq), dtype=torch.float32, device=dev)
    ctx = nat.default_context(0)
    s = torch.cuda.current_stream().cuda_stream
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ev = int(lengths.sum()) * n_freq
    out = {"workload": f"LS precision study: {n_curves} curves, lengths log-uniform [64, 16384] "
                       f"(mean {lengths.mean():.0f}), seasonal cadence 3000 d, {n_freq} "
                       "frequencies uniform in [0.01, 20] / d", "evals": ev, "folds": {}}
    for name, flags in (("plain (reference fold)", nat.PF_MODE_PLAIN),
                        ("chosen split-precision", nat.PF_MODE_CHOSEN),
                        ("chosen exact", nat.PF_MODE_CHOSEN | nat.PF_FOLD_EXACT),
                        ("all-FP32", nat.PF_MODE_CHOSEN | nat.PF_FOLD_F32)):
        def run(flags=flags):
            ctx.check(ctx.lib.pf_ls_dev(ctx.handle, d_t.data_ptr(), d_m.data_ptr(),
                                        off.ctypes.data, n_curves, d_p.data_ptr(), n_freq,
                                        d_d.data_ptr(), 1, flags, pg.data_ptr(), s))
        run()
        ms_ = _event_ms(torch, run, max(1, args.steps), flush)
        out["folds"][name] = {"ms": ms_, "evals_per_s": ev / (ms_ * 1e-3)}
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------- main


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--curves", type=int, default=N_CURVES)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    ap.add_argument("--workload", default="batch",
                    choices=["batch", "small", "ragged", "lsgrad", "precision", "fpw", "bls",
                             "device"],
                    help="'small': CE stats on 100 x 1024; 'ragged': the mixed ragged batch; "
                         "'lsgrad': LS derivatives and "
                         "Newton refinement; 'precision': LS folds on the precision-study "
                         "batch; 'fpw' / 'bls': FPW / BLS on the benchmark batch; 'device': "
                         "periodograms of "
                         "device-resident curves left on the GPU (separate reports, 1 GPU)")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.workload != "batch":
        {"small": small_arm, "ragged": ragged_arm, "lsgrad": lsgrad_arm,
         "precision": precision_arm, "fpw": fpw_arm, "bls": lambda a: fpw_arm(a, bls=True),
         "device": device_arm}[args.workload](args)
        return

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    # Each rank processes its own batch of curves (weak scaling, no exchange).
    ts, ms, periods, pdts = make_workload(args.curves, SEED + rank)
    from periodfind_b200 import _native as nat
    from periodfind_b200.distributed import max_over_ranks

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    pipes = measure_pipes() if rank == 0 else {}

    chosen = DeviceStep(ts, ms, periods, pdts, nat.PF_MODE_CHOSEN, torch, local)
    clocks = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    ms_step, launches = time_device(chosen, args.steps, args.warmup, torch, flush)
    clock_info = clocks.stop()
    ms_step = max_over_ranks(ms_step, device="cuda")
    ce_ms, aov_ms = time_kernels(chosen, torch)

    plain = DeviceStep(ts, ms, periods, pdts, nat.PF_MODE_PLAIN, torch, local)
    plain_ms, _ = time_device(plain, max(1, min(args.steps, 3)), 1, torch, flush)
    plain_ms = max_over_ranks(plain_ms, device="cuda")
    del plain

    e2e_s = time_e2e(ts, ms, periods, pdts, max(1, min(args.steps, 3)), 1, local)
    e2e_s = max_over_ranks(e2e_s, device="cuda")
    if dist:
        dist.barrier()

    n_eval = evals_per_step(args.curves) * world
    value = n_eval / (ms_step * 1e-3)
    if rank == 0:
        # Roofline of the dominant kernel (CE fold): FP64-pipe operations.
        evals_ce = args.curves * N_POINTS * N_PERIODS * len(PDTS)
        fp64_per_eval = FP64_OPS_PER_EVAL
        achieved = evals_ce * fp64_per_eval / (ce_ms * 1e-3) / 1e9
        peak = pipes.get("dfma", {}).get("per_s", float("nan")) / 1e9
        in_bytes = args.curves * N_POINTS * 8 + N_PERIODS * 4
        out_bytes = args.curves * N_PERIODS * len(PDTS) * 4
        hbm_gbs = (in_bytes + out_bytes) / (ce_ms * 1e-3) / 1e9
        cpu = None if args.no_cpu else cpu_baseline(ts, ms, periods, pdts)
        h2d = 2 * sum(t.nbytes + m.nbytes for t, m in zip(ts, ms)) + 2 * (periods.nbytes + pdts.nbytes)
        d2h = 2 * args.curves * N_PEAKS * 12
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 fold (exact), f32/fixed-point statistics", "data": "synthetic",
            "config": {"workload": WORKLOAD, "curves_per_gpu": args.curves,
                       "points": N_POINTS, "periods": N_PERIODS, "pdts": list(PDTS),
                       "l2": "flushed (256 MB write) between timed steps",
                       "parallelism": f"{world} independent replicas (curves sharded)"},
            "plain": {"value": n_eval / (plain_ms * 1e-3), "ms_per_step": plain_ms,
                      "chosen_over_plain": plain_ms / ms_step},
            "e2e": {"value": n_eval / e2e_s, "unit": "evals/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "ms_per_step": e2e_s * 1e3,
                    "path": "gpu.ConditionalEntropy/AOV.calc(list of numpy, output='peaks')"},
            "roofline": {"bound": "fp64", "kernel": "CE fold (chosen)",
                         "achieved": achieved, "peak": peak, "unit": "Gop/s",
                         "frac": achieved / peak if peak == peak else None,
                         "ops_per_eval": fp64_per_eval, "kernel_ms": ce_ms,
                         "peak_source": "measured DFMA rate (periodfind_b200/csrc/pipe_peaks.cu)",
                         "traffic": CE_TRAFFIC_BYTES,
                         "shared_atomic_view": {
                             "achieved_gops": evals_ce / (ce_ms * 1e-3) / 1e9,
                             "peak_gops": pipes.get("atoms_u32_private", {}).get("per_s", float("nan")) / 1e9,
                             "ops_per_eval": 1},
                         "hbm_view": {"achieved_gbs": hbm_gbs, "peak_gbs": 6453.7,
                                      "frac": hbm_gbs / 6453.7}},
            "kernels_ms": {"ce_fold": ce_ms, "aov_fold": aov_ms},
            "pipes": {k: round(v["per_s"] / 1e12, 3) for k, v in pipes.items()},
            "cpu_baseline": cpu,
            "clocks": clock_info,
            "gpu_launches": int(launches),
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


# FP64-pipe operations per evaluation in the chosen CE bin kernel's fast
# path: t * RN(1/P) (DMUL), floor (DADD.RD), bin with fraction bits
# (DFMA.RD), plus DMUL + DFMA for t - c t^2 on the period-derivative cells.
FP64_OPS_PER_EVAL = 3 + 2 * sum(1 for d in PDTS if d != 0.0) / len(PDTS)
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one
# full-size CE bin_kernel launch (1000 curves x 4096 points x 2e4 cells),
# from one ncu capture of this benchmark.
CE_TRAFFIC_BYTES = 52514048 + 28131328

if __name__ == "__main__":
    main()
