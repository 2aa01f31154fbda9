# cython: language_level=3, boundscheck=False, wraparound=False
"""Host-side helpers of the ctypes path, compiled because the Python route
costs more than the work it wraps.

curve_pointers: curve lengths and data addresses of a list of numpy arrays.
    Taking one array's address from Python (``a.ctypes.data``) costs about a
    microsecond; a batch of 100 000 light curves spent a fifth of a second
    per array list on it.  Here the addresses are read from the array
    structs.
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

