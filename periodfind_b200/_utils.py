"""Input preparation and validation for the periodogram classes.

Same behaviour and messages as the reference's periodfind/_utils.py:12-96
(prepare_magnitudes, validate_inputs, ensure_float32), so code that relies on
the reference's exceptions and warnings keeps working.
"""

import contextlib
import gc
import warnings

import numpy as np


@contextlib.contextmanager
def gc_paused():
    """Pause the cyclic garbage collector while a batch's result objects are
    built.  Tens of thousands of new objects trigger full collections whose
    cost grows with everything else the process holds (with torch imported,
    ~75 ms per 32 000 results against 13 ms paused); the results hold no
    reference cycles, so pausing loses nothing.  A collector that the caller
    had already disabled stays disabled."""
    was = gc.isenabled()
    gc.disable()
    try:
        yield
    finally:
        if was:
            gc.enable()


def prepare_magnitudes(mags, center, normalize):
    """Centre, normalise, or pass through magnitude arrays (float32 numpy).

    center:    m - mean(m)
    normalize: ((m - min) / (max - min)) * 0.999 + 5e-4, i.e. into (0, 1)
    Both set: warns and centres (periodfind/_utils.py:29-37).
    """
    if center and normalize:
        warnings.warn(
            "Center and normalize are conflicting settings. Normalize will be ignored.",
            RuntimeWarning,
            stacklevel=3,
        )
    if center:
        return _prepare_batch(mags, "pf_center_mags", _center_one)
    if normalize:
        return _prepare_batch(mags, "pf_normalize_mags", _normalize_one)
    return mags


def _center_one(mag):
    return mag - np.mean(mag)


def _normalize_one(mag):
    lo = np.min(mag)
    hi = np.max(mag)
    return ((mag - lo) / (hi - lo)) * 0.999 + 5e-4


def _prepare_batch(mags, native_fn, one):
    """Centre or normalise a whole batch in the native library
    (pf_center_mags / pf_normalize_mags): numpy's float32 arithmetic per
    curve, so every value equals numpy's one-curve-at-a-time result.
    Batches with an empty curve, or not all float32 1-D, take the per-curve
    numpy path `one` (and its warnings and errors)."""
    arrs = [np.asarray(m) for m in mags]
    if not arrs or any(a.ndim != 1 or a.size == 0 or a.dtype != np.float32 for a in arrs):
        return [one(mag) for mag in mags]
    # In the native library (multithreaded, same float32 arithmetic).
    from . import _native as nat

    n = len(arrs)
    lens = np.fromiter((a.shape[0] for a in arrs), dtype=np.uint64, count=n)
    starts = np.zeros(n, dtype=np.uint64)
    np.cumsum(lens[:-1], out=starts[1:])
    src, keep = nat.host_pointers(arrs, lens)
    flat = np.empty(int(lens.sum()), dtype=np.float32)
    dst = (np.uint64(flat.ctypes.data) + np.uint64(4) * starts).astype(np.uintp)
    rc = getattr(nat.load(), native_fn)(src.ctypes.data, lens.ctypes.data, n, dst.ctypes.data)
    del keep
    if rc != nat.PF_OK:
        raise RuntimeError(f"magnitude preparation failed ({rc})")
    bounds = starts.tolist() + [flat.shape[0]]
    return nat.FlatList([flat[a:b] for a, b in zip(bounds[:-1], bounds[1:])], flat, dst)


def validate_inputs(times, mags):
    """Raise ValueError unless times and mags pair up curve by curve."""
    if len(times) != len(mags):
        raise ValueError(
            f"times and mags must have the same number of light curves, "
            f"got {len(times)} and {len(mags)}"
        )
    for i, (t, m) in enumerate(zip(times, mags)):
        if len(t) != len(m):
            raise ValueError(
                f"times[{i}] and mags[{i}] have different lengths: {len(t)} vs {len(m)}"
            )


def ensure_float32(arrays, name):
    """Raise TypeError unless every array is float32."""
    for i, arr in enumerate(arrays):
        if arr.dtype != np.float32:
            raise TypeError(f"{name}[{i}] has dtype {arr.dtype}, expected float32")
