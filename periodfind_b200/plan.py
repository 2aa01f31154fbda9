"""Batch plans: the whole device pipeline for one fixed batch shape recorded
once as a CUDA graph and replayed (pf_plan_create / pf_plan_launch).

No counterpart in the reference, whose drivers copy, launch and synchronise
per call.  The plan keeps the device tensors it was made with: refill
`mags` (or `times`) in place and launch again to process the next batch of
the same shape.  Inputs are CSR device tensors as for the *_dev entry
points (float32 times / magnitudes, host int64 offsets)."""

from __future__ import annotations

import ctypes

import numpy as np

from . import _native as nat

_ALGOS = {"ce": nat.PF_ALGO_CE, "aov": nat.PF_ALGO_AOV, "ls": nat.PF_ALGO_LS}


class BatchPlan:
    def __init__(self, algo, times, mags, offsets, periods, period_dts, out, *, n_phase=10,
                 n_mag=10, phase_overlap=1, mag_overlap=1, flags=nat.PF_MODE_CHOSEN,
                 n_peaks=0, min_distance=1, peak_idx=None, peak_val=None, device=0):
        if algo not in _ALGOS:
            raise ValueError(f"algo must be one of {sorted(_ALGOS)}")
        self.lib = nat.load()
        self._keep = (times, mags, periods, period_dts, out, peak_idx, peak_val)
        self.offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        n_curves = len(self.offsets) - 1
        handle = ctypes.c_void_p()
        ptr = lambda t: t.data_ptr() if t is not None else None
        rc = self.lib.pf_plan_create(
            device, _ALGOS[algo], ptr(times), ptr(mags), self.offsets.ctypes.data, n_curves,
            ptr(periods), periods.numel(), ptr(period_dts), period_dts.numel(), n_phase, n_mag,
            phase_overlap, mag_overlap, flags, ptr(out), n_peaks, min_distance, ptr(peak_idx),
            ptr(peak_val), ctypes.byref(handle))
        if rc != nat.PF_OK:
            raise nat.PeriodfindError(rc, self.lib.pf_plan_error(None).decode())
        self.handle = handle

    def launch(self, stream=None):
        """Replay the graph on `stream` (a torch.cuda.Stream; None: the
        current torch stream)."""
        import torch

        s = (stream or torch.cuda.current_stream()).cuda_stream
        rc = self.lib.pf_plan_launch(self.handle, s)
        if rc != nat.PF_OK:
            raise nat.PeriodfindError(rc, self.lib.pf_plan_error(self.handle).decode())

    def close(self):
        if getattr(self, "handle", None):
            self.lib.pf_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        self.close()
