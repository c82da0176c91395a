"""Seeded synthetic inputs (numpy) from lib/libdtcgen.so.

The matrix families and value distributions are those of the benchmark
configurations; they stand in for the reference's dataset files, which are
not available here.
"""
import ctypes as C

import numpy as np

from ._lib import gen


class CSR:
    """Square-or-rectangular CSR matrix: rowptr int32[M+1], col int32[nnz], val float32[nnz]."""

    def __init__(self, rowptr, col, val, M, K):
        self.rowptr, self.col, self.val, self.M, self.K = rowptr, col, val, M, K

    @property
    def nnz(self):
        return int(self.rowptr[-1])


def _take(h):
    G = gen()
    M, K, nnz = C.c_int32(), C.c_int32(), C.c_int64()
    G.dtcgen_shape(h, C.byref(M), C.byref(K), C.byref(nnz))
    rowptr = np.empty(M.value + 1, np.int32)
    col = np.empty(nnz.value, np.int32)
    val = np.empty(nnz.value, np.float32)
    G.dtcgen_copy(h, rowptr.ctypes.data, col.ctypes.data, val.ctypes.data)
    G.dtcgen_free(h)
    return CSR(rowptr, col, val, M.value, K.value)


def uniform(M, K=None, mean=8.0, seed=0):
    """Row lengths Poisson(mean), columns uniform without replacement, values U(-1,1)."""
    return _take(gen().dtcgen_uniform(M, M if K is None else K, float(mean), seed))


def rmat(scale=20, edge_factor=16.0, a=0.57, b=0.19, c=0.19, seed=0):
    """R-MAT graph, symmetrised + self-loops + deduplicated, GCN-normalised values."""
    return _take(gen().dtcgen_rmat(scale, float(edge_factor), a, b, c, seed))


def stencil27(n=126, seed=0):
    """27-point stencil on an n^3 grid; values N(0,1), diagonal 27 + |off-diagonal row sum|."""
    return _take(gen().dtcgen_stencil27(n, seed))


def zipf(M, s=2.1, dmin=1, dmax=2000, seed=0):
    """Degrees Zipf(s) truncated to [dmin, dmax]; values U(0,1) row-normalised."""
    return _take(gen().dtcgen_zipf(M, float(s), dmin, dmax, seed))


def banded(M, bandwidth, fill=0.5, seed=0):
    return _take(gen().dtcgen_banded(M, bandwidth, float(fill), seed))


def blockdiag(M, block, degree, noise=0.05, seed=0):
    return _take(gen().dtcgen_blockdiag(M, block, degree, float(noise), seed))


def normal(rows, cols, seed=0):
    """Dense float32 [rows, cols] with N(0,1) entries (counter-based, thread-count independent)."""
    out = np.empty((rows, cols), np.float32)
    gen().dtcgen_normal(out.ctypes.data, out.size, seed)
    return out
