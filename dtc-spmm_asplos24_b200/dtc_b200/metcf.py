"""Torch-tensor front end over the C ABI (device memory from torch's allocator).

``convert`` is the ME-TCF conversion (reference: DTCSpMM.preprocess_gpu,
DTC-SpMM/DTCSpMM.cpp:313-359); ``spmm`` / ``spmm_balance`` are the
window-scheduled and strict-balance SpMM (run_DTCSpMM / run_DTCSpMM_balance,
DTCSpMM.cpp:117-178); ``spmm_ex`` takes any B storage form and precision.
All work runs in libdtcspmm.so on torch's current CUDA stream.
"""
import ctypes as C
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib
from ._lib import call


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


@dataclass
class METCF:
    """ME-TCF arrays on the device (reference names in comments)."""
    RowWindowOffset: torch.Tensor   # int32 [nwin+1]
    TCblockRowid: torch.Tensor      # int32 [T]
    TCblocktileId: torch.Tensor     # uint8 [nnz]
    TCblockoffset: torch.Tensor     # int32 [T+1]
    SparseAToX: torch.Tensor        # int32 [T*W]
    T: int
    blockPartition: torch.Tensor    # int32 [nwin]
    edgeToColumn: torch.Tensor      # int32 [nnz]
    edgeToRow: torch.Tensor         # int32 [nnz]
    M: int
    H: int
    W: int
    TCvalues: Optional[torch.Tensor] = None  # float32 [nnz] tile order

    @property
    def nwin(self):
        return self.RowWindowOffset.numel() - 1

    @property
    def nnz(self):
        return self.TCblocktileId.numel()


def convert(rowptr, col, M, H=16, W=8, values=None, device="cuda"):
    """CSR (int32 host or device tensors/arrays) -> METCF on `device`."""
    rowptr = torch.as_tensor(rowptr, dtype=torch.int32).to(device).contiguous()
    col = torch.as_tensor(col, dtype=torch.int32).to(device).contiguous()
    nnz = col.numel()
    nwin = (M + H - 1) // H
    i32 = dict(dtype=torch.int32, device=device)
    bp = torch.zeros(nwin, **i32)
    e2c = torch.zeros(nnz, **i32)
    e2r = torch.zeros(nnz, **i32)
    rwo = torch.zeros(nwin + 1, **i32)
    wsb = C.c_size_t()
    call("dtc_convert_workspace_bytes", M, nnz, H, W, C.byref(wsb))
    ws = torch.empty(max(wsb.value, 1), dtype=torch.uint8, device=device)
    T = C.c_int64()
    call("dtc_convert_count", _ptr(col), _ptr(rowptr), M, nnz, H, W, _ptr(bp), _ptr(e2c),
         _ptr(e2r), _ptr(rwo), _ptr(ws), wsb.value, C.byref(T), _stream())
    T = T.value
    rowid = torch.zeros(T, **i32)
    tile = torch.zeros(nnz, dtype=torch.uint8, device=device)
    toff = torch.zeros(T + 1, **i32)
    s2x = torch.zeros(T * W, **i32)
    tv = None
    vals = None
    if values is not None:
        vals = torch.as_tensor(values, dtype=torch.float32).to(device).contiguous()
        tv = torch.zeros(nnz, dtype=torch.float32, device=device)
    call("dtc_convert_fill", _ptr(col), _ptr(rowptr), M, nnz, H, W, _ptr(e2c), _ptr(e2r),
         _ptr(rwo), T, _ptr(rowid), _ptr(tile), _ptr(toff), _ptr(s2x), _ptr(vals), _ptr(tv),
         _ptr(ws), wsb.value, _stream())
    return METCF(rwo, rowid, tile, toff, s2x, T, bp, e2c, e2r, M, H, W, tv)


def spmm(m: METCF, B: torch.Tensor, use_values=True, out=None):
    """Window-scheduled SpMM (one launch). A = 1 when the METCF has no values."""
    B = B.contiguous()
    N = B.shape[1]
    C_ = out if out is not None else torch.empty((m.M, N), dtype=torch.float32, device=B.device)
    vals = m.TCvalues if use_values else None
    call("dtc_spmm", _ptr(m.RowWindowOffset), _ptr(m.TCblocktileId), _ptr(m.TCblockoffset),
         _ptr(m.SparseAToX), _ptr(vals), m.M, m.nwin, m.T, _ptr(B), N, _ptr(C_), _stream())
    return C_


def spmm_balance_workspace_bytes(m: METCF, N):
    wsb = C.c_size_t()
    call("dtc_spmm_balance_workspace_bytes", m.M, m.T, N, C.byref(wsb))
    return wsb.value


def spmm_balance(m: METCF, B: torch.Tensor, use_values=True, out=None, workspace=None):
    """Strict-balance SpMM from TCblockRowid (deterministic two-phase reduction)."""
    B = B.contiguous()
    N = B.shape[1]
    C_ = out if out is not None else torch.empty((m.M, N), dtype=torch.float32, device=B.device)
    wsb = spmm_balance_workspace_bytes(m, N)
    ws = workspace if workspace is not None else torch.empty(max(wsb, 1), dtype=torch.uint8,
                                                              device=B.device)
    vals = m.TCvalues if use_values else None
    call("dtc_spmm_balance", _ptr(m.TCblockRowid), _ptr(m.TCblocktileId), _ptr(m.TCblockoffset),
         _ptr(m.SparseAToX), _ptr(vals), m.M, m.T, _ptr(B), N, _ptr(C_), _ptr(ws),
         ws.numel(), _stream())
    return C_


def spmm_mma_sync(m: METCF, B: torch.Tensor, use_values=True, out=None):
    """Legacy-ISA (mma.sync) SpMM, for comparison and odd N."""
    B = B.contiguous()
    N = B.shape[1]
    C_ = out if out is not None else torch.empty((m.M, N), dtype=torch.float32, device=B.device)
    vals = m.TCvalues if use_values else None
    call("dtc_spmm_mma_sync", _ptr(m.RowWindowOffset), _ptr(m.TCblocktileId),
         _ptr(m.TCblockoffset), _ptr(m.SparseAToX), _ptr(vals), m.M, m.nwin, _ptr(B), N,
         _ptr(C_), _stream())
    return C_


def pack_b(B: torch.Tensor, fmt: int):
    """fp32 B -> storage planes of `fmt` (list of 1 or 2 uint8 tensors)."""
    B = B.contiguous()
    rows, N = B.shape
    b0, b1 = C.c_size_t(), C.c_size_t()
    call("dtc_bformat_bytes", fmt, rows, N, C.byref(b0), C.byref(b1))
    p0 = torch.empty(max(b0.value, 1), dtype=torch.uint8, device=B.device)
    p1 = torch.empty(max(b1.value, 1), dtype=torch.uint8, device=B.device) if b1.value else None
    call("dtc_pack_b", fmt, _ptr(B), rows, N, _ptr(p0), _ptr(p1), _stream())
    return [p0] if p1 is None else [p0, p1]


def pack_b_into(B: torch.Tensor, fmt: int, planes):
    """Re-pack B into existing planes (no allocation; usable inside graph capture)."""
    B = B.contiguous()
    rows, N = B.shape
    call("dtc_pack_b", fmt, _ptr(B), rows, N, _ptr(planes[0]),
         _ptr(planes[1]) if len(planes) > 1 else None, _stream())
    return planes


def spmm_ex_workspace_bytes(m: METCF, N, mode=0, grid=0):
    """Workspace bytes of spmm_ex for this schedule: the partial tiles of balance
    mode (required) and the chunk-queue region after them (optional: without it
    the kernels run one CTA per chunk instead of persistent CTAs)."""
    wsb = C.c_size_t()
    call("dtc_spmm_ex_workspace_bytes", m.M, m.T, N, m.H, mode, grid, C.byref(wsb))
    return wsb.value


def spmm_ex_launches(m: METCF, mode=0, grid=0, queue=True):
    """Kernels one spmm_ex call launches: the chunk-table kernel (when the
    workspace holds the chunk queue), the SpMM, and the partial-tile reduction
    in balance mode when the blocks are cut into more than one chunk."""
    if m.T == 0:
        return 0
    sms = torch.cuda.get_device_properties(m.RowWindowOffset.device).multi_processor_count
    G = min(grid if grid > 0 else 16 * sms, m.T)
    return (1 if queue else 0) + 1 + (1 if (mode == 1 and G > 1) else 0)


def spmm_ex(m: METCF, planes, fmt, N, precision, mode=0, grid=0, use_values=True, out=None,
            workspace=None, ntile=0):
    """SpMM with any B storage form (planes from pack_b), precision and schedule
    (mode 0 window / 1 balance, grid = chunks, ntile = 128-feature tiles per CTA),
    on ME-TCF arrays of window height 16 or 32 and block width 8 (or 16 at height
    16)."""
    dev = planes[0].device
    C_ = out if out is not None else torch.empty((m.M, N), dtype=torch.float32, device=dev)
    wsb = C.c_size_t()
    call("dtc_spmm_ex_workspace_bytes", m.M, m.T, N, m.H, mode, grid, C.byref(wsb))
    ws = workspace
    if ws is None and wsb.value:
        ws = torch.empty(wsb.value, dtype=torch.uint8, device=dev)
    vals = m.TCvalues if use_values else None
    call("dtc_spmm_ex", _ptr(m.RowWindowOffset), _ptr(m.TCblocktileId), _ptr(m.TCblockoffset),
         _ptr(m.SparseAToX), _ptr(vals), m.M, m.nwin, m.T, m.H, m.W, fmt, _ptr(planes[0]),
         _ptr(planes[1]) if len(planes) > 1 else None, N, precision, _ptr(C_), mode, grid,
         ntile, _ptr(ws), 0 if ws is None else ws.numel(), _stream())
    return C_


def spmm_fused(m: METCF, planes, fmt, N, precision, bias=None, relu=False, mode=0, grid=0,
               ntile=0, use_values=True, out=None, workspace=None):
    """spmm_ex with C = act(A*B + bias) fused into the store of C (GCN epilogue)."""
    dev = planes[0].device
    C_ = out if out is not None else torch.empty((m.M, N), dtype=torch.float32, device=dev)
    wsb = C.c_size_t()
    call("dtc_spmm_ex_workspace_bytes", m.M, m.T, N, m.H, mode, grid, C.byref(wsb))
    ws = workspace
    if ws is None and wsb.value:
        ws = torch.empty(wsb.value, dtype=torch.uint8, device=dev)
    vals = m.TCvalues if use_values else None
    bias = None if bias is None else bias.to(torch.float32).contiguous()
    call("dtc_spmm_fused", _ptr(m.RowWindowOffset), _ptr(m.TCblocktileId),
         _ptr(m.TCblockoffset), _ptr(m.SparseAToX), _ptr(vals), m.M, m.nwin, m.T, m.H, m.W, fmt,
         _ptr(planes[0]), _ptr(planes[1]) if len(planes) > 1 else None, N, precision, _ptr(bias),
         1 if relu else 0, _ptr(C_), mode, grid, ntile, _ptr(ws), 0 if ws is None else ws.numel(),
         _stream())
    return C_


def gcn_layer(m: METCF, H, W, bias=None, relu=True, fmt=0, precision=0, mode=0, grid=0):
    """One GCN layer act(Â (H W) + b): the dense H W on cuBLAS, then the SpMM with
    bias + ReLU fused into its epilogue (one pass over C instead of two)."""
    XW = torch.mm(H, W).contiguous()
    N = XW.shape[1]
    planes = [XW] if fmt == 0 else pack_b(XW, fmt)
    return spmm_fused(m, planes, fmt, N, precision, bias=bias, relu=relu, mode=mode, grid=grid)


def _relabel(name, rowptr, col, val, rows_out, extra):
    dev = rowptr.device
    rows_in = rowptr.numel() - 1
    nnz = col.numel()
    b = C.c_size_t()
    K = extra[0] if name == "dtc_transpose_csr" else rows_in
    call("dtc_relabel_workspace_bytes", rows_in, K, nnz, C.byref(b))
    ws = torch.empty(max(b.value, 1), dtype=torch.uint8, device=dev)
    rp = torch.empty(rows_out + 1, dtype=torch.int32, device=dev)
    co = torch.empty(max(nnz, 1), dtype=torch.int32, device=dev)
    vo = torch.empty(max(nnz, 1), dtype=torch.float32, device=dev)
    n = C.c_int64()
    if name == "dtc_permute_csr":
        call(name, _ptr(rowptr), _ptr(col), _ptr(val), rows_in, nnz, _ptr(extra[1]), _ptr(rp),
             _ptr(co), _ptr(vo), C.byref(n), _ptr(ws), ws.numel(), _stream())
    else:
        call(name, _ptr(rowptr), _ptr(col), _ptr(val), rows_in, K, nnz, _ptr(rp), _ptr(co),
             _ptr(vo), C.byref(n), _ptr(ws), ws.numel(), _stream())
    return rp, co[: n.value], vo[: n.value]


def permute_csr(rowptr, col, val, perm):
    """P A Pᵀ (perm[new] = old) as canonical CSR: (rowptr, col, val) device tensors.

    The GPU form of reordering/TCA_reorder.py:308-326 + the scipy CSR rebuild of
    scripts/DTCSpMM/dataset.py:38-44 (columns sorted, duplicates summed).
    """
    i32 = lambda t: t.to(torch.int32).contiguous()
    val = None if val is None else val.to(torch.float32).contiguous()
    return _relabel("dtc_permute_csr", i32(rowptr), i32(col), val, rowptr.numel() - 1,
                    (None, i32(perm)))


def transpose_csr(rowptr, col, val, num_cols):
    """Aᵀ as canonical CSR (num_cols rows): the operand of the backward product Aᵀ·G."""
    i32 = lambda t: t.to(torch.int32).contiguous()
    val = None if val is None else val.to(torch.float32).contiguous()
    return _relabel("dtc_transpose_csr", i32(rowptr), i32(col), val, num_cols, (num_cols,))


def device_status(clear=True):
    """Device-side error word (bit 0: wait timeout, bit 1: bad index skipped)."""
    f = C.c_uint32()
    call("dtc_device_status", C.byref(f), 1 if clear else 0)
    return f.value
