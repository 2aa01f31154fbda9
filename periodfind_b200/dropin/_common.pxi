# Shared by the drop-in modules ce / aov / ls / fpw / bls (included
# textually by each): the library context per device, per-curve pointers,
# one driver for every algorithm and output, and the result objects.
#
# The modules replace periodfind's own periodfind/{ce,aov,ls,fpw,bls}.pyx
# inside the periodfind package.  As the originals do, they take Statistics
# and Periodogram from that package and the input checks and magnitude
# preparation from its _utils (periodfind/ce.pyx:13-15), so the result
# objects are the package's own classes.

import numpy as np

cimport numpy as cnp
from libc.stdint cimport int64_t, uint32_t, uint64_t

from pf_abi cimport *

from periodfind import Periodogram, Statistics
from periodfind._utils import ensure_float32, prepare_magnitudes, validate_inputs

cnp.import_array()

N_PEAKS_DEFAULT = 32
MIN_DISTANCE_DEFAULT = 1

cdef enum Algo:
    ALGO_CE = 0
    ALGO_AOV = 1
    ALGO_LS = 2
    ALGO_FPW = 3
    ALGO_BLS = 4


cdef class _Context:
    """One pf_ctx (device buffers, pinned staging, stream, tuning cache)."""
    cdef pf_ctx* ptr

    def __cinit__(self, int device):
        cdef pf_ctx* c = NULL
        cdef int rc = pf_ctx_create(&c, device)
        if rc != PF_OK:
            # pf_last_error(NULL): the failed pf_ctx_create's message.
            raise RuntimeError(f"periodfind_b200 error {rc}: {pf_last_error(NULL).decode()}")
        self.ptr = c

    def __dealloc__(self):
        if self.ptr is not NULL:
            pf_ctx_destroy(self.ptr)


cdef dict _contexts = {}


cdef _Context _context(int device):
    c = _contexts.get(device)
    if c is None:
        c = _Context(device)
        _contexts[device] = c
    return <_Context>c


cdef int _check(pf_ctx* ctx, int rc) except -1:
    if rc != PF_OK:
        raise RuntimeError(f"periodfind_b200 error {rc}: {pf_last_error(ctx).decode()}")
    return 0


cdef class _Curves:
    """The data pointers (as uint64) of a list of float32 curves, with the
    contiguous arrays kept alive for the native call."""
    cdef readonly object ptrs
    cdef readonly list keep

    def __cinit__(self, list arrays):
        cdef Py_ssize_t i, n = len(arrays)
        self.ptrs = np.zeros(n, dtype=np.uint64)
        cdef uint64_t[::1] pv = self.ptrs
        cdef const float[::1] a
        self.keep = []
        for i in range(n):
            arr = np.ascontiguousarray(arrays[i], dtype=np.float32)
            self.keep.append(arr)
            if arr.shape[0] > 0:
                a = arr
                pv[i] = <uint64_t>&a[0]


cdef inline const float* const* _rows(uint64_t[::1] p):
    return <const float* const*>&p[0]


def _peak_statistics(idx, val, periods, period_dts, int n_peaks):
    """Per curve, its peaks as Statistics, best first, up to the first -1 --
    the objects the reference's CPU classes return for output='peaks'
    (periodfind/cpu/__init__.py:46-70)."""
    n_pdts = len(period_dts)
    valid = idx >= 0
    count = np.where(valid.all(axis=1), idx.shape[1], np.argmin(valid, axis=1)).tolist()
    safe = np.where(valid, idx, 0)
    per = np.asarray(periods)[safe // n_pdts].astype(np.float64).tolist()
    pdt = np.asarray(period_dts)[safe % n_pdts].astype(np.float64).tolist()
    vals = val.astype(np.float64).tolist()
    return [[Statistics([pr[k], dr[k]], vr[k], 0.0, 1.0, 0.0, 1.0) for k in range(c)]
            for pr, dr, vr, c in zip(per, pdt, vals, count)]


cdef object _calc(int algo, tuple params, int mode, int device, list times, list mags,
                  object errs, periods, period_dts, output, bint use_max, n_stats,
                  significance_type, n_peaks, min_distance):
    """Run one algorithm over the batch through the C ABI and build the
    requested output from the package's own result classes."""
    if output not in ("stats", "periodogram", "peaks"):
        raise NotImplementedError(
            f'Output type "{output}" is not implemented. '
            f'Use "stats", "periodogram" or "peaks".')
    cdef Py_ssize_t n = len(times)
    if n == 0:
        return []
    per = np.ascontiguousarray(periods, dtype=np.float32)
    pdt = np.ascontiguousarray(period_dts, dtype=np.float32)
    cdef uint64_t n_per = per.shape[0]
    cdef uint64_t n_pdt = pdt.shape[0]
    tc = _Curves(times)
    mc = _Curves(mags)
    lens = np.fromiter((len(t) for t in times), dtype=np.uint64, count=n)
    cdef uint64_t[::1] tp = tc.ptrs
    cdef uint64_t[::1] mp = mc.ptrs
    cdef uint64_t[::1] lv = lens
    cdef const float* const* T = _rows(tp)
    cdef const float* const* M = _rows(mp)
    cdef const float* const* E = NULL
    cdef uint64_t[::1] ep
    if errs is not None:
        ec = _Curves(list(errs))
        ep = ec.ptrs
        E = _rows(ep)
    cdef const float[::1] pv = per
    cdef const float[::1] dv = pdt
    cdef const float* P = &pv[0] if n_per > 0 else NULL
    cdef const float* D = &dv[0] if n_pdt > 0 else NULL
    cdef uint64_t nc = n
    cdef _Context ctx = _context(device)
    cdef pf_ctx* c = ctx.ptr
    # Integer parameters (bin counts, extents); BLS's qmin / qmax are floats.
    cdef uint32_t a0 = params[0] if len(params) > 0 else 0
    cdef uint32_t a1 = params[1] if len(params) > 1 and algo != ALGO_BLS else 0
    cdef uint32_t a2 = params[2] if len(params) > 2 and algo != ALGO_BLS else 0
    cdef uint32_t a3 = params[3] if len(params) > 3 else 0
    cdef float q0 = params[1] if algo == ALGO_BLS else 0.0
    cdef float q1 = params[2] if algo == ALGO_BLS else 0.0
    cdef int rc = PF_OK
    cdef uint32_t k, md
    cdef int64_t[:, ::1] iv
    cdef float[:, ::1] vv
    cdef int64_t* I
    cdef float* V
    cdef float[:, :, ::1] ov
    cdef float* O

    if output == "peaks":
        if int(n_peaks) < 0:
            raise ValueError("n_peaks must be >= 0")
        k = n_peaks
        md = min_distance
        idx = np.full((n, k), -1, dtype=np.int64)
        val = np.zeros((n, k), dtype=np.float32)
        if k > 0 and n_per * n_pdt > 0:
            iv = idx
            vv = val
            I = &iv[0, 0]
            V = &vv[0, 0]
            with nogil:
                if algo == ALGO_CE:
                    rc = pf_ce_peaks(c, T, M, &lv[0], nc, P, n_per, D, n_pdt, a0, a1, a2, a3,
                                     k, md, mode, I, V)
                elif algo == ALGO_AOV:
                    rc = pf_aov_peaks(c, T, M, &lv[0], nc, P, n_per, D, n_pdt, a0, a1, k, md,
                                      mode, I, V)
                elif algo == ALGO_LS:
                    rc = pf_ls_peaks(c, T, M, &lv[0], nc, P, n_per, D, n_pdt, k, md, mode, I, V)
                elif algo == ALGO_FPW:
                    rc = pf_fpw_peaks(c, T, M, E, &lv[0], nc, P, n_per, D, n_pdt, a0, k, md,
                                      mode, I, V)
                else:
                    rc = pf_bls_peaks(c, T, M, E, &lv[0], nc, P, n_per, D, n_pdt, a0, q0, q1,
                                      k, md, mode, I, V)
            _check(c, rc)
        return _peak_statistics(idx, val, periods, period_dts, k)

    out = np.zeros((n, n_per, n_pdt), dtype=np.float32)
    if n_per * n_pdt > 0:
        ov = out
        O = &ov[0, 0, 0]
        with nogil:
            if algo == ALGO_CE:
                rc = pf_ce(c, T, M, &lv[0], nc, P, n_per, D, n_pdt, a0, a1, a2, a3, mode, O)
            elif algo == ALGO_AOV:
                rc = pf_aov(c, T, M, &lv[0], nc, P, n_per, D, n_pdt, a0, a1, mode, O)
            elif algo == ALGO_LS:
                rc = pf_ls(c, T, M, &lv[0], nc, P, n_per, D, n_pdt, mode, O)
            elif algo == ALGO_FPW:
                rc = pf_fpw(c, T, M, E, &lv[0], nc, P, n_per, D, n_pdt, a0, mode, O)
            else:
                rc = pf_bls(c, T, M, E, &lv[0], nc, P, n_per, D, n_pdt, a0, q0, q1, mode, O)
        _check(c, rc)
    if output == "stats":
        return [Statistics.statistics_from_data(out[i], [periods, period_dts], use_max,
                                                n=n_stats, significance_type=significance_type)
                for i in range(n)]
    return [Periodogram(data, [periods, period_dts], use_max) for data in out]


cdef int _mode_flags(str mode) except -1:
    if mode == "chosen":
        return PF_MODE_CHOSEN
    if mode == "plain":
        return PF_MODE_PLAIN
    raise ValueError(f"mode must be 'chosen' or 'plain', got {mode!r}")


def _check_errs(times, errs):
    """The reference's checks of per-point uncertainties
    (periodfind/fpw.pyx:111-124): None means unit uncertainties."""
    if errs is None:
        return None
    ensure_float32(errs, 'errs')
    if len(errs) != len(times):
        raise ValueError(
            f"errs must have the same number of arrays as times, "
            f"got {len(errs)} and {len(times)}")
    for i, (e, t) in enumerate(zip(errs, times)):
        if len(e) != len(t):
            raise ValueError(
                f"errs[{i}] and times[{i}] have different lengths: "
                f"{len(e)} vs {len(t)}")
    return errs
