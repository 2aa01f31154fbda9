"""ctypes wrapper over the CPU oracle (oracle/oracle.c) and, when built, the
reference's own CUDA drivers (oracle/_ref/libpfref.so via ref_shim.cu).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py.  The periodfind_b200 product never imports it.

Every function takes curves as lists of float32 arrays (the reference's
calling convention, periodfind/ce.pyx:86-95) and returns float32 arrays of
shape [n_curves, n_periods, n_pdts] like the reference's Calc*Batched.
Magnitude preparation (normalize / center) is the caller's job, exactly as in
the reference, where the Cython wrapper prepares magnitudes before calling the
batched driver (periodfind/ce.pyx:167).
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_REF_PATH = os.path.join(HERE, "_ref", "libpfref.so")

_f32p = ctypes.POINTER(ctypes.c_float)
_f64p = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_u32p = ctypes.POINTER(ctypes.c_uint32)

_lib = None
_ref = None


def build() -> str:
    """Compile liboracle.so (the recipe is oracle/Makefile)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return _LIB_PATH


def _load():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
        os.path.join(HERE, "oracle.c")
    ):
        build()
    lib = ctypes.CDLL(_LIB_PATH)
    i64, u32, c_int = ctypes.c_int64, ctypes.c_uint32, ctypes.c_int
    lib.orc_ce_batched.argtypes = [_f32p, _f32p, _i64p, i64, _f32p, i64, _f32p, i64,
                                   u32, u32, u32, u32, c_int, c_int, _f32p]
    lib.orc_bls_batched.argtypes = [_f32p, _f32p, _f32p, _i64p, i64, _f32p, i64, _f32p, i64,
                                    ctypes.c_uint32, ctypes.c_float, ctypes.c_float, c_int,
                                    _f32p]
    lib.orc_fpw_batched.argtypes = [_f32p, _f32p, _f32p, _i64p, i64, _f32p, i64, _f32p, i64,
                                    ctypes.c_uint32, c_int, _f32p]
    lib.orc_aov_batched.argtypes = [_f32p, _f32p, _i64p, i64, _f32p, i64, _f32p, i64,
                                    u32, u32, c_int, c_int, _f32p]
    lib.orc_ls_batched.argtypes = [_f32p, _f32p, _i64p, i64, _f32p, i64, _f32p, i64,
                                   c_int, c_int, _f32p]
    lib.orc_ls_batched_f64.argtypes = [_f32p, _f32p, _i64p, i64, _f64p, i64, _f64p, i64,
                                       c_int, _f64p]
    lib.orc_aov_batched_f64.argtypes = [_f32p, _f32p, _i64p, i64, _f32p, i64, _f32p, i64,
                                        u32, u32, c_int, c_int, _f64p]
    lib.orc_phase_f64.argtypes = [_f32p, i64, _f64p, i64, ctypes.c_double, c_int, _f64p]
    lib.orc_ce_counts.argtypes = [_f32p, _f32p, i64, ctypes.c_float, ctypes.c_float,
                                  u32, u32, u32, u32, c_int, _u32p]
    lib.orc_ce_counts.restype = ctypes.c_float
    lib.orc_aov_counts.argtypes = [_f32p, _f32p, i64, ctypes.c_float, ctypes.c_float,
                                   u32, u32, c_int, _u32p]
    lib.orc_aov_counts.restype = ctypes.c_float
    lib.orc_find_top_peaks.argtypes = [_f32p, i64, i64, i64, c_int, _i64p, _f32p]
    lib.orc_find_top_peaks.restype = i64
    lib.orc_find_top_peaks_batched.argtypes = [_f32p, i64, i64, i64, i64, c_int, c_int,
                                               _i64p, _f32p]
    lib.orc_ls_derivs_f64.argtypes = [_f32p, _f32p, _i64p, i64, _f64p, i64, i64, c_int, _f64p]
    lib.orc_ls_grad_mags_f64.argtypes = [_f32p, _i64p, i64, _f64p, i64, i64, _f64p, c_int,
                                         _f64p]
    lib.orc_ls_refine_f64.argtypes = [_f32p, _f32p, _i64p, i64, _f64p, _f64p, i64, c_int,
                                      c_int, _f64p, _f64p]
    lib.orc_ls_power_tau_f64.argtypes = [_f64p, _f64p, i64, ctypes.c_double]
    lib.orc_ls_power_tau_f64.restype = ctypes.c_double
    _lib = lib
    return lib


def _ptr(a, t):
    return a.ctypes.data_as(t)


def pack(times, mags):
    """Concatenate per-curve arrays into CSR form (times, mags, offsets)."""
    if len(times) != len(mags):
        raise ValueError("times and mags must have the same number of curves")
    lens = np.array([len(t) for t in times], dtype=np.int64)
    offsets = np.zeros(len(times) + 1, dtype=np.int64)
    np.cumsum(lens, out=offsets[1:])
    t = (np.concatenate([np.asarray(x, np.float32) for x in times])
         if len(times) else np.zeros(0, np.float32))
    m = (np.concatenate([np.asarray(x, np.float32) for x in mags])
         if len(mags) else np.zeros(0, np.float32))
    return np.ascontiguousarray(t), np.ascontiguousarray(m), offsets


def _grid(periods, pdts):
    return (np.ascontiguousarray(periods, dtype=np.float32),
            np.ascontiguousarray(pdts, dtype=np.float32))


def ce(times, mags, periods, pdts, n_phase=10, n_mag=10, phase_overlap=1, mag_overlap=1,
       fused_tcorr=False, n_threads=0):
    """rust/src/ce.rs:39-116 batched as rust/src/lib.rs:31-88."""
    lib = _load()
    t, m, off = pack(times, mags)
    p, d = _grid(periods, pdts)
    out = np.zeros((len(off) - 1, len(p), len(d)), np.float32)
    lib.orc_ce_batched(_ptr(t, _f32p), _ptr(m, _f32p), _ptr(off, _i64p), len(off) - 1,
                       _ptr(p, _f32p), len(p), _ptr(d, _f32p), len(d), n_phase, n_mag,
                       phase_overlap, mag_overlap, int(fused_tcorr), n_threads,
                       _ptr(out, _f32p))
    return out


def fpw(times, mags, periods, pdts, n_bins=10, errs=None, n_threads=0):
    """rust/src/fpw.rs:12-66 batched as rust/src/lib.rs:202-256 (errs None:
    unit uncertainties, as periodfind/cpu/__init__.py:466-467)."""
    lib = _load()
    t, m, off = pack(times, mags)
    e = None
    if errs is not None:
        _, e, _ = pack(times, errs)
    p, d = _grid(periods, pdts)
    out = np.zeros((len(off) - 1, len(p), len(d)), np.float32)
    lib.orc_fpw_batched(_ptr(t, _f32p), _ptr(m, _f32p), None if e is None else _ptr(e, _f32p),
                        _ptr(off, _i64p), len(off) - 1, _ptr(p, _f32p), len(p), _ptr(d, _f32p),
                        len(d), n_bins, n_threads, _ptr(out, _f32p))
    return out


def bls(times, mags, periods, pdts, n_bins=50, qmin=0.01, qmax=0.5, errs=None, n_threads=0):
    """rust/src/bls.rs:19-134 batched as rust/src/lib.rs:264-322 (errs None:
    unit uncertainties)."""
    lib = _load()
    t, m, off = pack(times, mags)
    e = None
    if errs is not None:
        _, e, _ = pack(times, errs)
    p, d = _grid(periods, pdts)
    out = np.zeros((len(off) - 1, len(p), len(d)), np.float32)
    lib.orc_bls_batched(_ptr(t, _f32p), _ptr(m, _f32p), None if e is None else _ptr(e, _f32p),
                        _ptr(off, _i64p), len(off) - 1, _ptr(p, _f32p), len(p), _ptr(d, _f32p),
                        len(d), n_bins, qmin, qmax, n_threads, _ptr(out, _f32p))
    return out


def aov(times, mags, periods, pdts, n_phase=10, phase_overlap=1, fused_tcorr=False,
        n_threads=0):
    """rust/src/aov.rs:12-89 batched as rust/src/lib.rs:93-145."""
    lib = _load()
    t, m, off = pack(times, mags)
    p, d = _grid(periods, pdts)
    out = np.zeros((len(off) - 1, len(p), len(d)), np.float32)
    lib.orc_aov_batched(_ptr(t, _f32p), _ptr(m, _f32p), _ptr(off, _i64p), len(off) - 1,
                        _ptr(p, _f32p), len(p), _ptr(d, _f32p), len(d), n_phase,
                        phase_overlap, int(fused_tcorr), n_threads, _ptr(out, _f32p))
    return out


def aov_f64(times, mags, periods, pdts, n_phase=10, phase_overlap=1, fused_tcorr=False,
            n_threads=0):
    """AOV on the reference CPU path's bins with double sums and statistic."""
    lib = _load()
    t, m, off = pack(times, mags)
    p, d = _grid(periods, pdts)
    out = np.zeros((len(off) - 1, len(p), len(d)), np.float64)
    lib.orc_aov_batched_f64(_ptr(t, _f32p), _ptr(m, _f32p), _ptr(off, _i64p), len(off) - 1,
                            _ptr(p, _f32p), len(p), _ptr(d, _f32p), len(d), n_phase,
                            phase_overlap, int(fused_tcorr), n_threads, _ptr(out, _f64p))
    return out


def ls(times, mags, periods, pdts, fused_tcorr=False, n_threads=0):
    """rust/src/ls.rs:15-79 batched as rust/src/lib.rs:150-190."""
    lib = _load()
    t, m, off = pack(times, mags)
    p, d = _grid(periods, pdts)
    out = np.zeros((len(off) - 1, len(p), len(d)), np.float32)
    lib.orc_ls_batched(_ptr(t, _f32p), _ptr(m, _f32p), _ptr(off, _i64p), len(off) - 1,
                       _ptr(p, _f32p), len(p), _ptr(d, _f32p), len(d), int(fused_tcorr),
                       n_threads, _ptr(out, _f32p))
    return out


def ls_f64(times, mags, periods, pdts, n_threads=0):
    """All-double LS (exact oracle for precision studies); periods are taken as
    given (pass float32 periods to evaluate on the same grid as the kernels)."""
    lib = _load()
    t, m, off = pack(times, mags)
    p = np.ascontiguousarray(np.asarray(periods, dtype=np.float64))
    d = np.ascontiguousarray(np.asarray(pdts, dtype=np.float64))
    out = np.zeros((len(off) - 1, len(p), len(d)), np.float64)
    lib.orc_ls_batched_f64(_ptr(t, _f32p), _ptr(m, _f32p), _ptr(off, _i64p), len(off) - 1,
                           _ptr(p, _f64p), len(p), _ptr(d, _f64p), len(d), n_threads,
                           _ptr(out, _f64p))
    return out


def phase_f64(times, periods, period_dt=0.0, n_threads=0):
    """Exact folded phase frac((t - c t^2)/P) in double, shape [n_periods, n]."""
    lib = _load()
    t = np.ascontiguousarray(times, dtype=np.float32)
    p = np.ascontiguousarray(np.asarray(periods, dtype=np.float64))
    out = np.zeros((len(p), len(t)), np.float64)
    lib.orc_phase_f64(_ptr(t, _f32p), len(t), _ptr(p, _f64p), len(p), float(period_dt),
                      n_threads, _ptr(out, _f64p))
    return out


def _omega_arg(omega, n_curves):
    """(contiguous float64 omega, stride): [n_freq] -> stride 0, [n_curves, n_freq] -> n_freq."""
    w = np.ascontiguousarray(omega, dtype=np.float64)
    if w.ndim == 1:
        return w, 0, len(w)
    if w.ndim != 2 or w.shape[0] != n_curves:
        raise ValueError("omega must be [n_freq] or [n_curves, n_freq]")
    return w, w.shape[1], w.shape[1]


def ls_derivs_f64(times, mags, omega, n_threads=0):
    """FP64 LS power and omega-derivatives at angular frequencies `omega`
    ([n_freq] shared, or [n_curves, n_freq]).  Returns an array
    [n_curves, n_freq, 5] of (P, dP/dw, d2P/dw2, alpha, beta), times measured
    from the midpoint of each curve's time span."""
    lib = _load()
    t, m, off = pack(times, mags)
    n_curves = len(off) - 1
    w, stride, K = _omega_arg(omega, n_curves)
    out = np.zeros((n_curves, K, 5), np.float64)
    lib.orc_ls_derivs_f64(_ptr(t, _f32p), _ptr(m, _f32p), _ptr(off, _i64p), n_curves,
                          _ptr(w, _f64p), stride, K, n_threads, _ptr(out, _f64p))
    return out


def ls_grad_mags_f64(times, omega, gcoef, n_threads=0):
    """dL/dy for upstream-weighted coefficients gcoef [n_curves, n_freq, 2]
    (g * alpha, g * beta); returns the concatenated per-point gradient."""
    lib = _load()
    t, _, off = pack(times, times)
    n_curves = len(off) - 1
    w, stride, K = _omega_arg(omega, n_curves)
    g = np.ascontiguousarray(gcoef, dtype=np.float64)
    out = np.zeros(len(t), np.float64)
    lib.orc_ls_grad_mags_f64(_ptr(t, _f32p), _ptr(off, _i64p), n_curves, _ptr(w, _f64p),
                             stride, K, _ptr(g, _f64p), n_threads, _ptr(out, _f64p))
    return out


def ls_refine_f64(times, mags, omega0, half_width, n_steps=5, n_threads=0):
    """FP64 safeguarded Newton refinement of LS maxima from omega0
    [n_curves, K] within +-half_width; returns (omega, power), each [n_curves, K]."""
    lib = _load()
    t, m, off = pack(times, mags)
    n_curves = len(off) - 1
    w0 = np.ascontiguousarray(omega0, dtype=np.float64).reshape(n_curves, -1)
    hw = np.ascontiguousarray(half_width, dtype=np.float64).reshape(w0.shape)
    w = np.zeros_like(w0)
    p = np.zeros_like(w0)
    lib.orc_ls_refine_f64(_ptr(t, _f32p), _ptr(m, _f32p), _ptr(off, _i64p), n_curves,
                          _ptr(w0, _f64p), _ptr(hw, _f64p), w0.shape[1], int(n_steps),
                          n_threads, _ptr(w, _f64p), _ptr(p, _f64p))
    return w, p


def ls_power_tau_f64(t, y, omega):
    """The reference's tau expression in FP64 (FP64 times and magnitudes)."""
    lib = _load()
    t = np.ascontiguousarray(t, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    return lib.orc_ls_power_tau_f64(_ptr(t, _f64p), _ptr(y, _f64p), len(t), float(omega))


def ce_counts(t, m, period, pdt, n_phase=10, n_mag=10, po=1, mo=1, fused_tcorr=False):
    """(CE value, raw u32 histogram [n_phase, n_mag]) for one cell."""
    lib = _load()
    t = np.ascontiguousarray(t, np.float32)
    m = np.ascontiguousarray(m, np.float32)
    counts = np.zeros((n_phase, n_mag), np.uint32)
    v = lib.orc_ce_counts(_ptr(t, _f32p), _ptr(m, _f32p), len(t), float(period), float(pdt),
                          n_phase, n_mag, po, mo, int(fused_tcorr), _ptr(counts, _u32p))
    return v, counts


def aov_counts(t, m, period, pdt, n_phase=10, po=1, fused_tcorr=False):
    """(AOV value, raw u32 bin counts [n_phase]) for one cell."""
    lib = _load()
    t = np.ascontiguousarray(t, np.float32)
    m = np.ascontiguousarray(m, np.float32)
    counts = np.zeros(n_phase, np.uint32)
    v = lib.orc_aov_counts(_ptr(t, _f32p), _ptr(m, _f32p), len(t), float(period), float(pdt),
                           n_phase, po, int(fused_tcorr), _ptr(counts, _u32p))
    return v, counts


def find_top_peaks(data, n_peaks, min_distance, use_max):
    """rust/src/peaks.rs:228-238: (indices int64, values float32), trimmed."""
    lib = _load()
    d = np.ascontiguousarray(np.asarray(data, dtype=np.float32).ravel())
    n_peaks = int(n_peaks)
    idx = np.zeros(max(n_peaks, 1), np.int64)
    val = np.zeros(max(n_peaks, 1), np.float32)
    k = lib.orc_find_top_peaks(_ptr(d, _f32p), len(d), n_peaks, int(min_distance),
                               int(bool(use_max)), _ptr(idx, _i64p), _ptr(val, _f32p))
    return idx[:k].copy(), val[:k].copy()


def find_top_peaks_batched(data3d, n_peaks, min_distance, use_max, n_threads=0):
    """rust/src/lib.rs:508-548: idx [n_curves, n_peaks] (-1 padded), val (0 padded)."""
    lib = _load()
    d = np.ascontiguousarray(np.asarray(data3d, dtype=np.float32))
    nc = d.shape[0]
    flat = int(np.prod(d.shape[1:])) if d.ndim > 1 else 0
    idx = np.full((nc, n_peaks), -1, np.int64)
    val = np.zeros((nc, n_peaks), np.float32)
    lib.orc_find_top_peaks_batched(_ptr(d, _f32p), nc, flat, n_peaks, int(min_distance),
                                   int(bool(use_max)), n_threads, _ptr(idx, _i64p),
                                   _ptr(val, _f32p))
    return idx, val


# ----------------------------------------------------------- reference CUDA


def ref_available() -> bool:
    return os.path.exists(_REF_PATH)


def _load_ref():
    global _ref
    if _ref is not None:
        return _ref
    if not ref_available():
        raise FileNotFoundError(
            "oracle/_ref/libpfref.so is absent (build it with `make -C oracle ref` "
            "where the reference checkout exists)")
    lib = ctypes.CDLL(_REF_PATH)
    i64, u32 = ctypes.c_int64, ctypes.c_uint32
    lib.pfref_bls.argtypes = [_f32p, _f32p, _f32p, _i64p, i64, _f32p, i64, _f32p, i64, u32,
                              ctypes.c_float, ctypes.c_float, _f32p]
    lib.pfref_fpw.argtypes = [_f32p, _f32p, _f32p, _i64p, i64, _f32p, i64, _f32p, i64, u32,
                              _f32p]
    lib.pfref_ce.argtypes = [_f32p, _f32p, _i64p, i64, _f32p, i64, _f32p, i64,
                             u32, u32, u32, u32, _f32p]
    lib.pfref_aov.argtypes = [_f32p, _f32p, _i64p, i64, _f32p, i64, _f32p, i64,
                              u32, u32, _f32p]
    lib.pfref_ls.argtypes = [_f32p, _f32p, _i64p, i64, _f32p, i64, _f32p, i64, _f32p]
    _ref = lib
    return lib


def ref_cuda(algo, times, mags, periods, pdts, **kw):
    """Run the reference's own CUDA driver (built from its sources) on the GPU."""
    lib = _load_ref()
    t, m, off = pack(times, mags)
    p, d = _grid(periods, pdts)
    out = np.zeros((len(off) - 1, len(p), len(d)), np.float32)
    args = [_ptr(t, _f32p), _ptr(m, _f32p), _ptr(off, _i64p), len(off) - 1,
            _ptr(p, _f32p), len(p), _ptr(d, _f32p), len(d)]
    if algo == "ce":
        lib.pfref_ce(*args, kw.get("n_phase", 10), kw.get("n_mag", 10),
                     kw.get("phase_overlap", 1), kw.get("mag_overlap", 1), _ptr(out, _f32p))
    elif algo == "aov":
        lib.pfref_aov(*args, kw.get("n_phase", 10), kw.get("phase_overlap", 1),
                      _ptr(out, _f32p))
    elif algo == "ls":
        lib.pfref_ls(*args, _ptr(out, _f32p))
    elif algo == "bls":
        errs = kw.get("errs")
        e = (np.ones(len(t), np.float32) if errs is None
             else np.ascontiguousarray(np.concatenate(errs), np.float32))
        lib.pfref_bls(_ptr(t, _f32p), _ptr(m, _f32p), _ptr(e, _f32p), _ptr(off, _i64p),
                      len(off) - 1, _ptr(p, _f32p), len(p), _ptr(d, _f32p), len(d),
                      kw.get("n_bins", 50), kw.get("qmin", 0.01), kw.get("qmax", 0.5),
                      _ptr(out, _f32p))
    elif algo == "fpw":
        errs = kw.get("errs")
        e = (np.ones(len(t), np.float32) if errs is None
             else np.ascontiguousarray(np.concatenate(errs), np.float32))
        lib.pfref_fpw(_ptr(t, _f32p), _ptr(m, _f32p), _ptr(e, _f32p), _ptr(off, _i64p),
                      len(off) - 1, _ptr(p, _f32p), len(p), _ptr(d, _f32p), len(d),
                      kw.get("n_bins", 10), _ptr(out, _f32p))
    else:
        raise ValueError(algo)
    return out


def ref_fold_and_bin(algo, t, m, periods, pdts, n_phase=10, n_mag=10, po=1, mo=1):
    """The reference CUDA build's own bins for one curve, from its
    FoldAndBin step on the GPU (ConditionalEntropy::DeviceFoldAndBin,
    periodfind/cuda/ce.cu:262-290; AOV::DeviceFoldAndBin, aov.cu:265-299).

    CE: raw counts [n_per, n_pdt, n_phase * n_mag] uint32, recovered from
    the reference's count / (N * po * mo) floats (exact: the quotient is
    within 2 ulp of the true ratio and the counts are below 2^21).
    AOV: (counts [n_per, n_pdt, n_phase] uint32, sums, squared sums float32)
    exactly as the reference's AOVData holds them."""
    import torch

    lib = _load_ref()
    i64, u32, vp = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p
    lib.pfref_ce_hists.argtypes = [vp, vp, i64, vp, vp, i64, i64, u32, u32, u32, u32, vp]
    lib.pfref_aov_bins.argtypes = [vp, vp, i64, vp, vp, i64, i64, u32, u32, vp]
    dev = torch.device("cuda")
    cuda = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float32)).to(dev)
    d_t, d_m, d_p, d_d = cuda(t), cuda(m), cuda(periods), cuda(pdts)
    n, n_per, n_pdt = len(t), len(periods), len(pdts)
    if algo == "ce":
        h = np.zeros((n_per, n_pdt, n_phase * n_mag), np.float32)
        rc = lib.pfref_ce_hists(d_t.data_ptr(), d_m.data_ptr(), n, d_p.data_ptr(),
                                d_d.data_ptr(), n_per, n_pdt, n_phase, n_mag, po, mo,
                                h.ctypes.data)
        if rc != 0:
            raise RuntimeError("reference FoldAndBin failed")
        div = float(n * po * mo)
        counts = np.rint(h.astype(np.float64) * div).astype(np.uint32)
        return counts
    raw = np.zeros((n_per, n_pdt, n_phase, 3), np.uint32)
    rc = lib.pfref_aov_bins(d_t.data_ptr(), d_m.data_ptr(), n, d_p.data_ptr(), d_d.data_ptr(),
                            n_per, n_pdt, n_phase, po, raw.ctypes.data)
    if rc != 0:
        raise RuntimeError("reference FoldAndBin failed")
    return (raw[..., 0].copy(), raw[..., 1].copy().view(np.float32),
            raw[..., 2].copy().view(np.float32))
