"""Input preparation and validation for the periodogram classes.

Same behaviour and messages as the reference's periodfind/_utils.py:12-96
(prepare_magnitudes, validate_inputs, ensure_float32), so code that relies on
the reference's exceptions and warnings keeps working.
"""

import warnings

import numpy as np


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
        return [mag - np.mean(mag) for mag in mags]
    if normalize:
        return _normalize_batch(mags)
    return mags


def _normalize_batch(mags):
    """The per-curve normalisation over the whole batch at once: the same
    elementwise float32 expression and exact per-curve min / max, so every
    value equals the one-curve-at-a-time result.  Batches with an empty
    curve, or not all float32 1-D, take the per-curve path (and its errors)."""
    arrs = [np.asarray(m) for m in mags]
    if not arrs or any(a.ndim != 1 or a.size == 0 or a.dtype != np.float32 for a in arrs):
        out = []
        for mag in mags:
            lo = np.min(mag)
            hi = np.max(mag)
            out.append(((mag - lo) / (hi - lo)) * 0.999 + 5e-4)
        return out
    lens = np.fromiter((a.size for a in arrs), dtype=np.int64, count=len(arrs))
    flat = np.concatenate(arrs)
    starts = np.zeros(len(arrs), dtype=np.int64)
    np.cumsum(lens[:-1], out=starts[1:])
    lo = np.repeat(np.minimum.reduceat(flat, starts), lens)
    hi = np.repeat(np.maximum.reduceat(flat, starts), lens)
    res = ((flat - lo) / (hi - lo)) * 0.999 + 5e-4
    return np.split(res, starts[1:])


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
