"""ORACLE -- test infrastructure only (the checker, never the product path).

numpy/ctypes front end of ``oracle/metcf_oracle.c``: the CPU restatement of the
reference's ME-TCF conversion (DTC-SpMM/DTCSpMM_kernel.cu:107-419,
DTC-SpMM/DTCSpMM.cpp:313-359) and FP64/FP32 CSR SpMM. Only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this module.
"""
import ctypes
import os

import numpy as np

from . import build_oracle  # noqa: F401  (package-relative when imported as oracle.oracle)

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = build_oracle.build()
        _lib = ctypes.CDLL(path)
        i32p = ctypes.POINTER(ctypes.c_int32)
        _lib.oracle_metcf_num_blocks.restype = ctypes.c_int64
        _lib.oracle_metcf.restype = ctypes.c_int
        _lib.oracle_metcf_values.restype = ctypes.c_int
        del i32p
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _csr(rowptr, col):
    return (np.ascontiguousarray(rowptr, dtype=np.int32),
            np.ascontiguousarray(col, dtype=np.int32))


def metcf(rowptr, col, M, H=16, W=8, values=None):
    """Reference-exact ME-TCF arrays for a CSR matrix (dict of numpy arrays).

    Keys follow the reference tuple (DTCSpMM.cpp:356-358) plus the in-place
    outputs: RowWindowOffset, TCblockRowid, TCblocktileId, TCblockoffset,
    SparseAToX, T, blockPartition, edgeToColumn, edgeToRow, and TCvalues when
    ``values`` is given.
    """
    L = lib()
    rowptr, col = _csr(rowptr, col)
    nnz = int(rowptr[M])
    nwin = (M + H - 1) // H
    T = int(L.oracle_metcf_num_blocks(_p(rowptr), _p(col), ctypes.c_int32(M),
                                      ctypes.c_int32(H), ctypes.c_int32(W)))
    out = dict(
        blockPartition=np.zeros(nwin, np.int32),
        edgeToColumn=np.zeros(nnz, np.int32),
        edgeToRow=np.zeros(nnz, np.int32),
        RowWindowOffset=np.zeros(nwin + 1, np.int32),
        TCblockRowid=np.zeros(T, np.int32),
        TCblocktileId=np.zeros(nnz, np.uint8),
        TCblockoffset=np.zeros(T + 1, np.int32),
        SparseAToX=np.zeros(T * W, np.int32),
    )
    rc = L.oracle_metcf(_p(rowptr), _p(col), ctypes.c_int32(M), ctypes.c_int32(H),
                        ctypes.c_int32(W), _p(out["blockPartition"]), _p(out["edgeToColumn"]),
                        _p(out["edgeToRow"]), _p(out["RowWindowOffset"]),
                        _p(out["TCblockRowid"]), _p(out["TCblocktileId"]),
                        _p(out["TCblockoffset"]), _p(out["SparseAToX"]), ctypes.c_int64(T))
    if rc != 0:
        raise RuntimeError(f"oracle_metcf failed ({rc})")
    out["T"] = T
    if values is not None:
        v = np.ascontiguousarray(values, dtype=np.float32)
        tv = np.zeros(nnz, np.float32)
        L.oracle_metcf_values(_p(rowptr), _p(col), _p(v), ctypes.c_int32(M), ctypes.c_int32(H),
                              ctypes.c_int32(W), _p(out["edgeToColumn"]), _p(out["edgeToRow"]),
                              _p(out["RowWindowOffset"]), _p(out["TCblockoffset"]), _p(tv))
        out["TCvalues"] = tv
    return out


def spmm_f64(rowptr, col, values, M, B):
    """FP64 CSR SpMM; ``values=None`` = the reference's implicit A = 1."""
    rowptr, col = _csr(rowptr, col)
    B = np.ascontiguousarray(B, dtype=np.float32)
    N = B.shape[1]
    C = np.empty((M, N), np.float64)
    v = None if values is None else np.ascontiguousarray(values, dtype=np.float32)
    lib().oracle_spmm_f64(_p(rowptr), _p(col), None if v is None else _p(v),
                          ctypes.c_int32(M), ctypes.c_int32(N), _p(B), _p(C))
    return C


def spmm_absbound_f64(rowptr, col, values, M, B):
    """sum_e |A[i,e]| |B[col_e, j]| per output element (tolerance scale)."""
    rowptr, col = _csr(rowptr, col)
    B = np.ascontiguousarray(B, dtype=np.float32)
    N = B.shape[1]
    C = np.empty((M, N), np.float64)
    v = None if values is None else np.ascontiguousarray(values, dtype=np.float32)
    lib().oracle_spmm_absbound_f64(_p(rowptr), _p(col), None if v is None else _p(v),
                                   ctypes.c_int32(M), ctypes.c_int32(N), _p(B), _p(C))
    return C


def spmm_f32(rowptr, col, values, M, B, nthreads=0, out=None):
    """Host FP32 CSR SpMM over ``nthreads`` OpenMP threads (the CPU baseline)."""
    rowptr, col = _csr(rowptr, col)
    B = np.ascontiguousarray(B, dtype=np.float32)
    N = B.shape[1]
    C = out if out is not None else np.empty((M, N), np.float32)
    v = None if values is None else np.ascontiguousarray(values, dtype=np.float32)
    lib().oracle_spmm_f32(_p(rowptr), _p(col), None if v is None else _p(v),
                          ctypes.c_int32(M), ctypes.c_int32(N), _p(B), _p(C),
                          ctypes.c_int(nthreads))
    return C


def metcf_spmm_f64(m, M, B, H=16, W=8, tc_values=None):
    """FP64 product straight from ME-TCF arrays (tile semantics of the reference)."""
    B = np.ascontiguousarray(B, dtype=np.float32)
    N = B.shape[1]
    C = np.empty((M, N), np.float64)
    tv = None if tc_values is None else np.ascontiguousarray(tc_values, dtype=np.float32)
    lib().oracle_metcf_spmm_f64(_p(m["RowWindowOffset"]), _p(m["TCblocktileId"]),
                                _p(m["TCblockoffset"]), _p(m["SparseAToX"]),
                                None if tv is None else _p(tv), ctypes.c_int32(M),
                                ctypes.c_int32(H), ctypes.c_int32(W), ctypes.c_int32(N),
                                _p(B), _p(C))
    return C


def pack_split24(B):
    """fp32 -> (bf16 hi plane, u8 extension plane), RNE at 16 significant bits."""
    B = np.ascontiguousarray(B, dtype=np.float32)
    hi = np.empty(B.shape, np.uint16)
    ext = np.empty(B.shape, np.uint8)
    lib().oracle_pack_split24(_p(B), ctypes.c_int64(B.size), _p(hi), _p(ext))
    return hi, ext


def pack_bf16(B):
    B = np.ascontiguousarray(B, dtype=np.float32)
    out = np.empty(B.shape, np.uint16)
    lib().oracle_pack_bf16(_p(B), ctypes.c_int64(B.size), _p(out))
    return out


def pack_bf16x2(B):
    """BF16X2 planes: hi = bf16_rn(b), lo = bf16_rn(b - hi) (the difference is
    exact in fp32), lo = 0 where hi is not finite. Returns (hi, lo) uint16."""
    B = np.ascontiguousarray(B, dtype=np.float32)
    hi = pack_bf16(B)
    hf = (hi.astype(np.uint32) << 16).view(np.float32)
    with np.errstate(invalid="ignore", over="ignore"):
        d = np.where(np.isfinite(hf), B - hf, np.float32(0)).astype(np.float32)
    return hi, pack_bf16(d)


def bf16x2_values(hi, lo):
    """hi + lo as float64 (the value the BF16X2 planes stand for)."""
    f = lambda u: (u.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    return f(hi) + f(lo)


def pack_fp8(B):
    """fp32 rows -> (e4m3 bytes, fp32 per-row scales)."""
    B = np.ascontiguousarray(B, dtype=np.float32)
    rows, N = B.shape
    q = np.empty(B.shape, np.uint8)
    s = np.empty(rows, np.float32)
    lib().oracle_pack_fp8(_p(B), ctypes.c_int64(rows), ctypes.c_int32(N), _p(q), _p(s))
    return q, s


def e4m3_values(q):
    """float32 values of an array of e4m3 bytes."""
    L = lib()
    L.oracle_e4m3_value.restype = ctypes.c_float
    L.oracle_e4m3_value.argtypes = [ctypes.c_uint8]
    table = np.array([L.oracle_e4m3_value(i) for i in range(256)], np.float32)
    return table[q]


def split24_values(hi, ext):
    """fp32 values of the 24-bit form (the B the split kernels multiply)."""
    u = (hi.astype(np.uint32) << 16) | (ext.astype(np.uint32) << 8)
    return u.view(np.float32)


def permute_csr(rowptr, col, val, perm):
    """P A Pᵀ as canonical CSR, restating reordering/TCA_reorder.py:308-326
    (reorder[i_new] = i_old; d[old] = new; src' = d[src], dst' = d[dst]) and
    the CSR rebuild of scripts/DTCSpMM/dataset.py:38-44 (scipy coo -> csr:
    columns sorted per row, duplicates summed). Duplicates are summed in input
    CSR order; ``val=None`` counts every entry as 1 like the reference."""
    rowptr = np.asarray(rowptr, np.int64)
    col = np.asarray(col, np.int64)
    perm = np.asarray(perm, np.int64)
    M = len(rowptr) - 1
    if sorted(perm.tolist()) != list(range(M)):
        raise ValueError("perm is not a permutation")
    d = np.empty(M, np.int64)
    d[perm] = np.arange(M)
    src = np.repeat(np.arange(M), np.diff(rowptr))
    return _coo_to_csr(d[src], d[col], val, M, M)


def transpose_csr(rowptr, col, val, K):
    """Aᵀ (K rows) as canonical CSR, duplicates summed in input CSR order."""
    rowptr = np.asarray(rowptr, np.int64)
    col = np.asarray(col, np.int64)
    M = len(rowptr) - 1
    src = np.repeat(np.arange(M), np.diff(rowptr))
    return _coo_to_csr(col, src, val, K, M)


def _coo_to_csr(r, c, val, rows, cols):
    nnz = len(r)
    v = np.ones(nnz, np.float32) if val is None else np.asarray(val, np.float32)
    order = np.lexsort((np.arange(nnz), c, r))  # stable by (row, col)
    r, c, v = r[order], c[order], v[order]
    first = np.ones(nnz, bool)
    first[1:] = (r[1:] != r[:-1]) | (c[1:] != c[:-1])
    starts = np.flatnonzero(first)
    out_v = np.empty(len(starts), np.float32)
    ends = np.append(starts[1:], nnz)
    for k, (s, e) in enumerate(zip(starts, ends)):  # sequential float32 sums
        acc = np.float32(v[s])
        for j in range(s + 1, e):
            acc = np.float32(acc + v[j])
        out_v[k] = acc
    out_r, out_c = r[starts], c[starts]
    rp = np.zeros(rows + 1, np.int64)
    np.add.at(rp, out_r + 1, 1)
    return np.cumsum(rp).astype(np.int32), out_c.astype(np.int32), out_v
