"""Graph files in the reference's .npz layout (scripts/DTCSpMM/dataset.py:21-44):
arrays ``src_li``, ``dst_li`` (one entry per edge) and ``num_nodes``. Loading
builds the CSR on the GPU with dtc_coo_to_csr, with the reference's semantics:
every edge has value 1, duplicate edges sum, columns are sorted within rows."""
import ctypes as C

import numpy as np
import torch

from ._lib import call
from .metcf import _ptr, _stream


def coo_to_csr(src, dst, num_rows, num_cols=None, val=None, device="cuda"):
    """(rowptr, col, val) device tensors of the canonical CSR of a COO edge list."""
    num_cols = num_rows if num_cols is None else num_cols
    s = torch.as_tensor(np.asarray(src, np.int32) if not torch.is_tensor(src) else src)
    d = torch.as_tensor(np.asarray(dst, np.int32) if not torch.is_tensor(dst) else dst)
    s = s.to(device, torch.int32).contiguous()
    d = d.to(device, torch.int32).contiguous()
    v = None if val is None else torch.as_tensor(val).to(device, torch.float32).contiguous()
    nnz = s.numel()
    b = C.c_size_t()
    call("dtc_relabel_workspace_bytes", num_rows, num_cols, nnz, C.byref(b))
    ws = torch.empty(max(b.value, 1), dtype=torch.uint8, device=device)
    rp = torch.empty(num_rows + 1, dtype=torch.int32, device=device)
    co = torch.empty(max(nnz, 1), dtype=torch.int32, device=device)
    vo = torch.empty(max(nnz, 1), dtype=torch.float32, device=device)
    n = C.c_int64()
    call("dtc_coo_to_csr", _ptr(s), _ptr(d), _ptr(v), num_rows, num_cols, nnz, _ptr(rp), _ptr(co),
         _ptr(vo), C.byref(n), _ptr(ws), ws.numel(), _stream())
    return rp, co[: n.value], vo[: n.value]


def load_npz(path, device="cuda"):
    """(rowptr, col, val, num_nodes) of an .npz graph file (val = edge multiplicity)."""
    z = np.load(path)
    n = int(z["num_nodes"])
    rp, col, val = coo_to_csr(z["src_li"], z["dst_li"], n, device=device)
    return rp, col, val, n


def save_npz(path, src, dst, num_nodes):
    """Writes an edge list in the same layout."""
    np.savez(path, src_li=np.asarray(src, np.int64), dst_li=np.asarray(dst, np.int64),
             num_nodes=np.int64(num_nodes))
