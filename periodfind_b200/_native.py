"""ctypes binding of the C ABI in include/pf.h (libpfb200.so, built in-tree).

There is no fallback: if the library is missing or no B200 is present, the
GPU classes raise.  Build with `python -m periodfind_b200.build`.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

from . import _host

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpfb200.so")

PF_OK = 0
PF_EINVAL = -1
PF_ECUDA = -2
PF_ENOMEM = -3
PF_EUNSUPPORTED = -4
PF_ETIMEOUT = -5

PF_MODE_PLAIN = 0x0
PF_MODE_CHOSEN = 0x1
PF_SEM_CPU = 0x10
PF_FOLD_F32 = 0x100
PF_FOLD_DF = 0x200
PF_FOLD_EXACT = 0x400
PF_TIMING = 0x1000
PF_REF_STATS = 0x2000
PF_NO_TUNE = 0x4000
PF_ASYNC = 0x8000
PF_TRIG_SINCOS = 0x10000
PF_TRIG_RECURRENCE = 0x20000
PF_BINS_SHARED = 0x40000
PF_ONE_LAUNCH = 0x80000
PF_HOST_NORMALIZE = 0x100000
PF_HOST_CENTER = 0x200000
PF_PREP_CENTER, PF_PREP_NORMALIZE = 1, 2
PF_ALGO_CE, PF_ALGO_AOV, PF_ALGO_LS = 0, 1, 2

_vp = ctypes.c_void_p
_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32
_int = ctypes.c_int
_f32 = ctypes.c_float

# Every symbol the header declares, with its argument types.
SIGNATURES = {
    "pf_version": ([], _int),
    "pf_ctx_create": ([ctypes.POINTER(_vp), _int], _int),
    "pf_ctx_destroy": ([_vp], None),
    "pf_last_error": ([_vp], ctypes.c_char_p),
    "pf_ce": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _u32, _u32, _int,
               _vp], _int),
    "pf_aov": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _int, _vp], _int),
    "pf_ls": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _int, _vp], _int),
    "pf_ls_fgrid": ([_vp, _vp, _vp, _vp, _u64, ctypes.c_double, ctypes.c_double, _u64, _int,
                     _vp], _int),
    "pf_ls_fgrid_dev": ([_vp, _vp, _vp, _vp, _u64, ctypes.c_double, ctypes.c_double, _u64,
                         _int, _vp, _vp], _int),
    "pf_bin_counts": ([_vp, _int, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _u32,
                       _u32, _int, _vp, _vp], _int),
    "pf_ce_peaks": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _u32, _u32,
                     _u32, _u32, _int, _vp, _vp], _int),
    "pf_aov_peaks": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _u32, _u32,
                      _int, _vp, _vp], _int),
    "pf_ls_peaks": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _int, _vp,
                     _vp], _int),
    "pf_wait": ([_vp], _int),
    "pf_prepare_mags_dev": ([_vp, _vp, _vp, _u64, _int, _vp, _vp], _int),
    "pf_bls": ([_vp, _vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _f32, _f32, _int,
                _vp], _int),
    "pf_bls_peaks": ([_vp, _vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _f32, _f32,
                      _u32, _u32, _int, _vp, _vp], _int),
    "pf_fpw": ([_vp, _vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _int, _vp], _int),
    "pf_fpw_peaks": ([_vp, _vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _u32,
                      _int, _vp, _vp], _int),
    "pf_ce_stats": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _u32, _u32,
                     _u32, _int, _vp, _vp, _vp], _int),
    "pf_aov_stats": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _u32, _int,
                      _vp, _vp, _vp], _int),
    "pf_ls_stats": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _int, _vp, _vp, _vp],
                    _int),
    "pf_find_peaks": ([_vp, _vp, _u64, _u64, _u32, _u32, _int, _vp, _vp], _int),
    "pf_ce_dev": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _u32, _u32, _int,
                   _vp, _vp], _int),
    "pf_aov_dev": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _int, _vp, _vp],
                   _int),
    "pf_ls_dev": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _int, _vp, _vp], _int),
    "pf_find_peaks_dev": ([_vp, _vp, _u64, _u64, _u32, _u32, _int, _vp, _vp, _vp], _int),
    "pf_ls_peaks_dev_noalloc": ([_vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _int,
                                 _vp, _vp, _vp, ctypes.c_char_p, _u64], _int),
    "pf_curve_latency": ([_vp, _u64, _vp], _int),
    "pf_fold_phase_dev": ([_vp, _int, _vp, _u64, _vp, _u64, ctypes.c_float, _vp, _vp], _int),
    "pf_ls_eval_dev": ([_vp, _vp, _vp, _vp, _u64, _vp, _u64, _u64, _vp, _vp, _vp, _vp, _vp],
                       _int),
    "pf_ls_backward_dev": ([_vp, _vp, _vp, _u64, _vp, _u64, _u64, _vp, _vp, _vp, _vp, _vp,
                            _vp], _int),
    "pf_ls_refine_dev": ([_vp, _vp, _vp, _vp, _u64, _vp, _vp, _u64, _u32, _vp, _vp, _vp], _int),
    "pf_tuning_report": ([_vp, ctypes.c_char_p, _u64], _int),
    "pf_normalize_mags": ([_vp, _vp, _u64, _vp], _int),
    "pf_center_mags": ([_vp, _vp, _u64, _vp], _int),
    "pf_plan_create": ([_int, _int, _vp, _vp, _vp, _u64, _vp, _u64, _vp, _u64, _u32, _u32, _u32,
                        _u32, _int, _vp, _u32, _u32, _vp, _vp, ctypes.POINTER(_vp)], _int),
    "pf_plan_launch": ([_vp, _vp], _int),
    "pf_plan_error": ([_vp], ctypes.c_char_p),
    "pf_plan_destroy": ([_vp], None),
    "pf_plan_kernel_count": ([_vp], _u64),
    "pf_launch_count": ([_vp], _u64),
    "pf_last_kernel_ms": ([_vp], ctypes.c_double),
}

_lib = None
_lib_lock = threading.Lock()


class PeriodfindError(RuntimeError):
    """A failure reported by the native library (status code + message)."""

    def __init__(self, code, message):
        super().__init__(f"periodfind_b200 error {code}: {message}")
        self.code = code


def load():
    """Load libpfb200.so and declare its signatures (raises if absent)."""
    global _lib
    with _lib_lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is not built; run `python -m periodfind_b200.build` "
                "(there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
        return lib


class Context:
    """One native context (device buffers, stream, pinned staging).

    Calls on one Context are serialised with a lock; the native call itself
    runs without the GIL (ctypes releases it).
    """

    def __init__(self, device: int = 0):
        self.lib = load()
        h = _vp()
        rc = self.lib.pf_ctx_create(ctypes.byref(h), int(device))
        if rc != PF_OK:
            raise PeriodfindError(rc, self.lib.pf_last_error(None).decode())
        self.handle = h
        self.device = device
        self.lock = threading.Lock()

    def close(self):
        if getattr(self, "handle", None):
            self.lib.pf_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def tuning_report(self) -> str:
        """The autotuner's choices on this context (pf_tuning_report)."""
        buf = ctypes.create_string_buffer(1 << 16)
        self.check(min(0, self.lib.pf_tuning_report(self.handle, buf, len(buf))))
        return buf.value.decode()

    def check(self, rc):
        if rc != PF_OK:
            raise PeriodfindError(rc, self.lib.pf_last_error(self.handle).decode())

    @property
    def launches(self) -> int:
        return int(self.lib.pf_launch_count(self.handle))

    @property
    def last_kernel_ms(self) -> float:
        return float(self.lib.pf_last_kernel_ms(self.handle))


_contexts: dict = {}
_ctx_lock = threading.Lock()


def default_context(device: int = 0) -> Context:
    with _ctx_lock:
        ctx = _contexts.get(device)
        if ctx is None:
            ctx = Context(device)
            _contexts[device] = ctx
        return ctx


class FlatList(list):
    """A list of float32 curves that are consecutive views of one buffer,
    with their data pointers already computed (what the batch magnitude
    preparation returns).  Slices keep the pointers."""

    def __init__(self, arrays, buf, ptrs):
        super().__init__(arrays)
        self.buf = buf
        self.ptrs = ptrs

    def __getitem__(self, k):
        if isinstance(k, slice) and self.ptrs is not None:
            return FlatList(list.__getitem__(self, k), self.buf, self.ptrs[k])
        return list.__getitem__(self, k)


def _dropping_pointers(name):
    # A change to the list itself makes the stored pointers stale: forget
    # them, and the curves are then addressed one by one.
    base = getattr(list, name)

    def method(self, *args, **kwargs):
        self.ptrs = None
        return base(self, *args, **kwargs)

    method.__name__ = name
    return method


for _name in ("__setitem__", "__delitem__", "__iadd__", "__imul__", "append", "extend",
              "insert", "pop", "remove", "reverse", "sort", "clear"):
    setattr(FlatList, _name, _dropping_pointers(_name))


def host_pointers(arrs, lengths):
    """Data pointers (uintp) of float32 curves, and the object that keeps
    them valid.  1-D contiguous float32 arrays are used in place (their
    addresses read by the compiled helper); otherwise short curves are
    gathered into one buffer, whose pointers are arithmetic (taking an
    array's address from Python costs about a microsecond, more than copying
    a thousand points), and longer ones converted one by one."""
    n = len(lengths)
    if isinstance(arrs, FlatList) and arrs.ptrs is not None and len(arrs.ptrs) == n:
        return arrs.ptrs, arrs
    if n:
        ptrs = np.empty(n, dtype=np.uintp)
        lens = np.empty(n, dtype=np.uint64)
        if _host.curve_pointers(arrs, lens, ptrs) and np.array_equal(lens, lengths):
            return ptrs, arrs
    total = int(lengths.sum()) if n else 0
    if 0 < n and total <= 1024 * n and total <= (1 << 22):
        buf = np.concatenate(arrs).astype(np.float32, copy=False)
        starts = np.zeros(n, dtype=np.uint64)
        np.cumsum(lengths[:-1], out=starts[1:])
        return (np.uint64(buf.ctypes.data) + np.uint64(4) * starts).astype(np.uintp), buf
    keep = [np.ascontiguousarray(a, dtype=np.float32) for a in arrs]
    return np.fromiter((a.ctypes.data for a in keep), dtype=np.uintp, count=n), keep


class CurveBatch:
    """Per-curve host pointers and lengths for the host-pointer entry points.

    Keeps references to the (contiguous float32) data so the pointers stay
    valid for the duration of the native call.
    """

    def __init__(self, times, mags):
        n = len(times)
        self.n = n
        if n and len(mags) == n and not isinstance(mags, FlatList):
            # Arrays used in place, lengths and addresses read in one pass.
            lt, lm = np.empty(n, dtype=np.uint64), np.empty(n, dtype=np.uint64)
            pt, pm = np.empty(n, dtype=np.uintp), np.empty(n, dtype=np.uintp)
            if _host.curve_pointers(times, lt, pt) and _host.curve_pointers(mags, lm, pm):
                if not np.array_equal(lt, lm):
                    raise ValueError("times and mags must have the same length for every curve")
                self.lengths = lt
                self.tptr, self._times = pt, times
                self.mptr, self._mags = pm, mags
                return
        self.lengths = np.fromiter((len(t) for t in times), dtype=np.uint64, count=n)
        mlen = np.fromiter((len(m) for m in mags), dtype=np.uint64, count=len(mags))
        if not np.array_equal(mlen, self.lengths):
            raise ValueError("times and mags must have the same length for every curve")
        self.tptr, self._times = host_pointers(times, self.lengths)
        self.mptr, self._mags = host_pointers(mags, self.lengths)

    def args(self):
        return (self.tptr.ctypes.data, self.mptr.ctypes.data, self.lengths.ctypes.data, self.n)


def ptr(a) -> int:
    return a.ctypes.data
