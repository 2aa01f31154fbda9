"""Separate reports of bench.py (--workload batch / small / lsgrad /
precision / fpw / bls / device), one JSON object each, on one GPU.  Every
timed region carries its own nvidia-smi clock record ("clocks").

  batch      CE(10x10) + AOV(15) + top-32 peaks, 1000 curves x 4096 points x
             10000 log periods [0.1, 100] d x pdts [0, 1e-6]: chosen and
             plain device steps, end-to-end calc(output='peaks')
  small      CE 10x10 'stats' on 100 curves x 1024 points x 1000 periods
  lsgrad     LS derivatives and Newton refinement, 2000 x 2048 x 20000
  precision  LS folds on the precision-study batch (10000 ragged curves x
             50000 frequencies)
  fpw / bls  FPW(10) / BLS(50, 0.01, 0.5) on the 1000 x 4096 batch
  device     device-resident CE + AOV periodograms against the host path
  profile    a short run whose kernels ncu captures (NVTX range pf_profile):
             chosen CE / AOV / LS on a sample of the ragged batch
  profile_batch  the same for chosen CE and AOV on the 1000 x 4096 batch
             shape (default 10 curves)
"""

from __future__ import annotations

import os
import time

import numpy as np

import lightcurves as lc
from bench import (N_CURVES, N_PEAKS, N_PERIODS, N_POINTS, PDTS, SEED, BatchStep, Clocks,
                   make_workload, time_steps)


def _emit(out, clocks):
    import json

    out["clocks"] = clocks.union()
    out["clocks_regions"] = clocks.regions
    print(json.dumps(out), flush=True)


def batch_arm(args):
    """The 1000 x 4096 batch: chosen and plain device steps and the public
    calc(output='peaks') path from numpy lists."""
    import torch

    from periodfind_b200 import _native as nat
    from periodfind_b200 import gpu

    torch.cuda.set_device(0)
    clocks = Clocks(0)
    ts, ms, periods, pdts = make_workload(args.curves or N_CURVES)
    n = len(ts)
    ev = 2 * n * N_POINTS * N_PERIODS * len(PDTS)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()
    out = {"workload": f"CE(10x10) + AOV(15) + top-32 peaks, {n} curves x {N_POINTS} points x "
                       f"{N_PERIODS} log periods [0.1, 100] d x pdts {list(PDTS)}", "evals": ev}
    for mode, flags in (("chosen", nat.PF_MODE_CHOSEN), ("plain", nat.PF_MODE_PLAIN)):
        st = BatchStep(ts, ms, periods, pdts, flags, torch, 0)
        with clocks.region(mode):
            ms_, _ = time_steps(st.run, max(1, args.steps), 2, torch, flush, stream)
        out[mode] = {"ms_per_step": ms_, "evals_per_s": ev / (ms_ * 1e-3)}
        st.ctx.close()
    out["chosen_over_plain"] = out["plain"]["ms_per_step"] / out["chosen"]["ms_per_step"]
    ce, aov = gpu.ConditionalEntropy(10, 10), gpu.AOV(15)
    run = lambda: (ce.calc(ts, ms, periods, pdts, output="peaks", n_peaks=N_PEAKS),
                   aov.calc(ts, ms, periods, pdts, output="peaks", n_peaks=N_PEAKS))
    run()
    w = []
    with clocks.region("e2e_calc"):
        for _ in range(max(1, min(args.steps, 3))):
            t0 = time.perf_counter()
            run()
            w.append(time.perf_counter() - t0)
    out["e2e_calc"] = {"ms_per_step": float(np.mean(w)) * 1e3, "evals_per_s": ev / np.mean(w),
                       "path": "gpu.ConditionalEntropy/AOV.calc(list of numpy, output='peaks')"}
    _emit(out, clocks)


def fpw_arm(args, bls=False):
    """FPW(10) -- or, with bls, BoxLeastSquares(50, 0.01, 0.5) -- over the
    benchmark batch (1000 curves x 4096 points, 10000 log periods in
    [0.1, 100] d x pdts [0, 1e-6]) with per-point uncertainties U[0.02, 0.1]:
    device time of the chosen and plain forms (the kernel, CUDA events),
    end-to-end calc(output='peaks') from numpy lists, and the oracle (the
    Rust path's restatement) on all host cores over a sample."""
    from periodfind_b200 import gpu

    clocks = Clocks(0)
    ts, ms, periods, pdts = make_workload(args.curves or N_CURVES)
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
        with clocks.region(f"{mode}_kernel"):
            for _ in range(max(3, args.steps)):
                obj.periodograms(ts, ms, periods, pdts, errs=es)
                k.append(ctx.lib.pf_last_kernel_ms(ctx.handle))
        kms = float(np.median(k))
        obj.calc(ts, ms, periods, pdts, errs=es, output="peaks", n_peaks=N_PEAKS)
        w = []
        with clocks.region(f"{mode}_e2e"):
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
    _emit(out, clocks)



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
    clocks = Clocks(0)
    ts, ms, periods, pdts = make_workload(args.curves or N_CURVES)
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
        with clocks.region(name):
            for _ in range(max(3, args.steps)):
                t0 = time.perf_counter()
                fn()
                w.append(time.perf_counter() - t0)
        ms_ = float(np.median(w)) * 1e3
        out[name] = {"ms": ms_, "evals_per_s": evals / (ms_ * 1e-3)}
    _emit(out, clocks)



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
    clocks = Clocks(0)
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
        # Each timed loop runs for at least a second so that the clock
        # record (200 ms samples) covers it.
        k = []
        with clocks.region(f"{mode}_kernel"):
            t_end = time.perf_counter() + 1.0
            while len(k) < max(3, args.steps) or time.perf_counter() < t_end:
                run()
                torch.cuda.synchronize()
                k.append(ctx.lib.pf_last_kernel_ms(ctx.handle))
        obj = gpu.ConditionalEntropy(10, 10, mode=mode)
        obj.calc(ts, ms, periods, pdts, output="stats")
        w = []
        with clocks.region(f"{mode}_e2e"):
            t_end = time.perf_counter() + 1.0
            while len(w) < max(3, args.steps) or time.perf_counter() < t_end:
                t0 = time.perf_counter()
                obj.calc(ts, ms, periods, pdts, output="stats")
                w.append(time.perf_counter() - t0)
        kms, ws = float(np.median(k)), float(np.median(w))
        out[mode] = {"kernel_ms": kms, "evals_per_s": evals / (kms * 1e-3),
                     "e2e_ms": ws * 1e3, "e2e_evals_per_s": evals / ws}
    # End to end through the C ABI from the host arrays (no Python result
    # objects): pf_ce_stats with the normalisation fused into the packing,
    # statistics and best cells back in host arrays.
    bt = nat.CurveBatch(ts, ms)
    st = np.empty((n_curves, 4), np.float32)
    bi = np.empty((n_curves, 1), np.int64)
    bv = np.empty((n_curves, 1), np.float32)

    def cabi():
        ctx.check(ctx.lib.pf_ce_stats(ctx.handle, *bt.args(), periods.ctypes.data, len(periods),
                                      pdts.ctypes.data, 1, 10, 10, 1, 1, 1,
                                      nat.PF_MODE_CHOSEN | nat.PF_HOST_NORMALIZE,
                                      st.ctypes.data, bi.ctypes.data, bv.ctypes.data))
    for _ in range(3):
        cabi()
    w = []
    with clocks.region("chosen_e2e_cabi"):
        t_end = time.perf_counter() + 1.0
        while len(w) < max(3, args.steps) or time.perf_counter() < t_end:
            t0 = time.perf_counter()
            cabi()
            w.append(time.perf_counter() - t0)
    out["chosen"]["e2e_cabi_ms"] = float(np.median(w)) * 1e3
    out["chosen"]["e2e_cabi_evals_per_s"] = evals / float(np.median(w))
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
    _emit(out, clocks)



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
    clocks = Clocks(0)
    n_curves, n_pts, n_freq = 2000, 2048, 20000
    t, m, off = lc.seasonal_ls_batch(np.full(n_curves, n_pts), SEED + 4)
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
    with clocks.region("grid_periodogram_peaks"):
        ms_grid = _event_ms(torch, grid_peaks, reps, flush)
    with clocks.region("autograd_forward"):
        ms_fwd = _event_ms(torch, forward, reps, flush)
    ms_bwd = []
    with clocks.region("autograd_backward"):
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
    with clocks.region("newton_refine"):
        ms_ref = _event_ms(torch, refine, max(reps, 200), flush)
    ev_ref = n_curves * n_pts * N_PEAKS * 6
    out["grid_periodogram_peaks"] = {"ms": ms_grid, "evals_per_s": ev / (ms_grid * 1e-3)}
    out["autograd_forward"] = {"ms": ms_fwd, "evals_per_s": ev / (ms_fwd * 1e-3)}
    out["autograd_backward"] = {"ms": ms_bwd, "evals_per_s": ev / (ms_bwd * 1e-3)}
    out["newton_refine_5_steps"] = {"ms": ms_ref, "evals_per_s": ev_ref / (ms_ref * 1e-3),
                                    "peaks": n_curves * N_PEAKS}
    _emit(out, clocks)


def precision_arm(args):
    """10000 curves, lengths log-uniform in [64, 16384], seasonal cadence over
    3000 days; 50000 frequencies uniform in [0.01, 20] / day.  Times the LS
    periodogram with each fold: plain (the reference's FP64-divide fold),
    chosen split-precision, chosen exact, and the all-FP32 fold."""
    import torch

    from periodfind_b200 import _native as nat

    torch.cuda.set_device(0)
    clocks = Clocks(0)
    rng = np.random.default_rng(SEED + 3)
    n_curves = args.curves or 10000
    lengths = np.exp(rng.uniform(np.log(64), np.log(16384), n_curves)).astype(np.int64)
    t, m, off = lc.seasonal_ls_batch(lengths, SEED + 3)
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
        with clocks.region(name):
            ms_ = _event_ms(torch, run, max(1, args.steps), flush)
        out["folds"][name] = {"ms": ms_, "evals_per_s": ev / (ms_ * 1e-3)}
    # The same grid given as a uniform frequency grid (pf_ls_fgrid_dev):
    # trial frequency k is exactly 0.01 + k * df.  Sincos per evaluation,
    # the angle-addition recurrence along the grid, and the autotuner's pick
    # per length class.
    f_min, df = 0.01, (20.0 - 0.01) / (n_freq - 1)
    for name, flags in (("frequency grid, sincos", nat.PF_MODE_CHOSEN | nat.PF_TRIG_SINCOS),
                        ("frequency grid, recurrence",
                         nat.PF_MODE_CHOSEN | nat.PF_TRIG_RECURRENCE),
                        ("frequency grid, tuned trig", nat.PF_MODE_CHOSEN)):
        def run(flags=flags):
            ctx.check(ctx.lib.pf_ls_fgrid_dev(ctx.handle, d_t.data_ptr(), d_m.data_ptr(),
                                              off.ctypes.data, n_curves, f_min, df, n_freq,
                                              flags, pg.data_ptr(), s))
        run()
        with clocks.region(name):
            ms_ = _event_ms(torch, run, max(1, args.steps), flush)
        out["folds"][name] = {"ms": ms_, "evals_per_s": ev / (ms_ * 1e-3)}
    out["tuning"] = [ln for ln in ctx.tuning_report().splitlines() if "fgrid" in ln]
    _emit(out, clocks)


def profile_arm(args):
    """A short run for ncu captures: the mixed ragged batch (--curves,
    default 10000), one tuned direct call per computation outside the
    capture, then inside the NVTX range "pf_profile" one chosen call each
    of CE, AOV and LS over the 20000 log periods, and LS on the uniform
    frequency grid of 20000 frequencies in [0.002, 20] / d with the sincos
    form and with the recurrence (4 or 5 class launches each).  Prints the
    kernel times (the library's CUDA events)."""
    import json

    import torch

    from bench import RaggedStep, ragged_grid
    from periodfind_b200 import _native as nat

    torch.cuda.set_device(0)
    n_curves = args.curves or 10000
    t, m, off = lc.ragged_batch(n_curves, SEED + 5)
    periods, pdts = ragged_grid()
    step = RaggedStep(t, m, off, periods, pdts, torch, 0, plans=False)
    c, lib = step.ctx, step.ctx.lib
    f_min, n_freq = 0.002, 20000
    df = (20.0 - f_min) / (n_freq - 1)
    fg = torch.empty((step.n, n_freq), dtype=torch.float32, device="cuda")

    def fgrid(flags):
        c.check(lib.pf_ls_fgrid_dev(c.handle, step.d_t.data_ptr(), step.mags["ls"].data_ptr(),
                                    step.off.ctypes.data, step.n, f_min, df, n_freq, flags,
                                    fg.data_ptr(), step.s))

    runs = [(a, lambda a=a: step.direct(a, nat.PF_MODE_CHOSEN, peaks=False))
            for a in ("ce", "aov", "ls")]
    runs += [("ls_fgrid_sincos", lambda: fgrid(nat.PF_MODE_CHOSEN | nat.PF_TRIG_SINCOS)),
             ("ls_fgrid_recurrence",
              lambda: fgrid(nat.PF_MODE_CHOSEN | nat.PF_TRIG_RECURRENCE))]
    for _, fn in runs:  # tuning and warm-up, outside the captured range
        fn()
    torch.cuda.synchronize()
    out = {"workload": f"ragged batch sample: {n_curves} curves ({int(off[-1])} points), "
                       f"{len(periods)} log periods / {n_freq} uniform frequencies",
           "kernel_ms": {}}
    torch.cuda.nvtx.range_push("pf_profile")
    for name, fn in runs:
        fn()
        torch.cuda.synchronize()
        out["kernel_ms"][name] = c.last_kernel_ms
    torch.cuda.nvtx.range_pop()
    out["tuning"] = c.tuning_report().strip().splitlines()
    step.close()
    print(json.dumps(out), flush=True)


def profile_batch_arm(args):
    """A short run for ncu captures on the 1000 x 4096 batch's shape
    (--curves, default 10): one tuned chosen call of CE and of AOV outside
    the capture, then inside the NVTX range "pf_profile" one chosen call of
    each (one class launch each: every curve has 4096 points).  Prints the
    kernel times (the library's CUDA events)."""
    import json

    import torch

    from periodfind_b200 import _native as nat

    torch.cuda.set_device(0)
    ts, ms, periods, pdts = make_workload(args.curves or 10)
    st = BatchStep(ts, ms, periods, pdts, nat.PF_MODE_CHOSEN, torch, 0)
    c, lib, h = st.ctx, st.ctx.lib, st.ctx.handle

    def common(m):
        return (h, st.t.data_ptr(), m.data_ptr(), st.off.ctypes.data, st.n, st.P.data_ptr(),
                st.np_, st.D.data_ptr(), st.nd)

    runs = [("ce", lambda: c.check(lib.pf_ce_dev(*common(st.m_ce), 10, 10, 1, 1,
                                                 nat.PF_MODE_CHOSEN, st.pg[0].data_ptr(),
                                                 st.s))),
            ("aov", lambda: c.check(lib.pf_aov_dev(*common(st.m_aov), 15, 1, nat.PF_MODE_CHOSEN,
                                                   st.pg[1].data_ptr(), st.s)))]
    for _, fn in runs:  # tuning and warm-up, outside the captured range
        fn()
    torch.cuda.synchronize()
    out = {"workload": f"{st.n} curves x {N_POINTS} points x {N_PERIODS} log periods x "
                       f"pdts {list(PDTS)}", "kernel_ms": {}}
    torch.cuda.nvtx.range_push("pf_profile")
    for name, fn in runs:
        fn()
        torch.cuda.synchronize()
        out["kernel_ms"][name] = c.last_kernel_ms
    torch.cuda.nvtx.range_pop()
    out["tuning"] = c.tuning_report().strip().splitlines()
    c.close()
    print(json.dumps(out), flush=True)


ARMS = {"batch": batch_arm, "profile": profile_arm, "profile_batch": profile_batch_arm, "small": small_arm, "lsgrad": lsgrad_arm,
        "precision": precision_arm, "fpw": fpw_arm, "bls": lambda a: fpw_arm(a, bls=True),
        "device": device_arm}


