# cython: language_level=3, boundscheck=False, wraparound=False
"""Host-side helpers of the ctypes path, compiled because the Python route
costs more than the work it wraps.

curve_pointers: curve lengths and data addresses of a list of numpy arrays.
    Taking one array's address from Python (``a.ctypes.data``) costs about a
    microsecond; a batch of 100 000 light curves spent a fifth of a second
    per array list on it.  Here the addresses are read from the array
    structs.

curve_check: whether a batch already has the form the native calls take
    (what validate_inputs, ensure_float32 and the fused magnitude
    preparation otherwise check one array at a time in Python).
"""

cimport numpy as cnp
import numpy as np

cnp.import_array()


def curve_pointers(arrs, cnp.uint64_t[::1] lengths, size_t[::1] pointers):
    """Write len(a) and the data address of every array of `arrs` into
    `lengths` and `pointers` (each at least len(arrs) long).  Returns False,
    leaving the outputs partly written, as soon as an entry is not a 1-D
    C-contiguous float32 numpy array (the caller then takes the general
    path, which converts)."""
    cdef Py_ssize_t i, n = len(arrs)
    cdef cnp.ndarray a
    if lengths.shape[0] < n or pointers.shape[0] < n:
        raise ValueError("output arrays are shorter than the curve list")
    seq = arrs if isinstance(arrs, (list, tuple)) else list(arrs)
    for i in range(n):
        o = seq[i]
        if not isinstance(o, cnp.ndarray):
            return False
        a = <cnp.ndarray>o
        if (cnp.PyArray_NDIM(a) != 1 or cnp.PyArray_TYPE(a) != cnp.NPY_FLOAT32
                or not cnp.PyArray_IS_C_CONTIGUOUS(a)):
            return False
        lengths[i] = <cnp.uint64_t>cnp.PyArray_DIM(a, 0)
        pointers[i] = <size_t>cnp.PyArray_DATA(a)
    return True



def curve_check(times, mags):
    """2 if `times` and `mags` are lists (or tuples) of equal length whose
    entries are 1-D C-contiguous float32 numpy arrays, pairwise of equal
    length, with no empty magnitude array; 1 if all that holds but some
    magnitude array is empty; 0 otherwise (the caller then runs the full
    checks, which raise the reference's exceptions)."""
    cdef Py_ssize_t i, n
    cdef cnp.ndarray a, b
    cdef int state = 2
    if not isinstance(times, (list, tuple)) or not isinstance(mags, (list, tuple)):
        return 0
    n = len(times)
    if len(mags) != n:
        return 0
    for i in range(n):
        o, p = times[i], mags[i]
        if not isinstance(o, cnp.ndarray) or not isinstance(p, cnp.ndarray):
            return 0
        a = <cnp.ndarray>o
        b = <cnp.ndarray>p
        if (cnp.PyArray_NDIM(a) != 1 or cnp.PyArray_NDIM(b) != 1
                or cnp.PyArray_TYPE(a) != cnp.NPY_FLOAT32 or cnp.PyArray_TYPE(b) != cnp.NPY_FLOAT32
                or not cnp.PyArray_IS_C_CONTIGUOUS(a) or not cnp.PyArray_IS_C_CONTIGUOUS(b)
                or cnp.PyArray_DIM(a, 0) != cnp.PyArray_DIM(b, 0)):
            return 0
        if cnp.PyArray_DIM(b, 0) == 0:
            state = 1
    return state
