"""Row reordering: the TCA clustering permutation (dtc_tca_reorder) and its
application (dtc_permute_csr), the GPU form of reordering/TCA_reorder.py and
the CSR rebuild of scripts/DTCSpMM/dataset.py:38-44."""
import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import TcaParams, call
from .metcf import _ptr, _stream, permute_csr


def default_params(**overrides):
    p = TcaParams()
    _lib.lib().dtc_tca_default_params(C.byref(p))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def tca_perm(rowptr, col, num_nodes, params=None):
    """perm[new] = old (int32 device tensor) for a square CSR on the device."""
    rowptr = rowptr.to(torch.int32).contiguous()
    col = col.to(torch.int32).contiguous()
    p = params if params is not None else default_params()
    b = C.c_size_t()
    call("dtc_tca_workspace_bytes", num_nodes, col.numel(), C.byref(p), C.byref(b))
    ws = torch.empty(max(b.value, 1), dtype=torch.uint8, device=rowptr.device)
    perm = torch.empty(max(num_nodes, 1), dtype=torch.int32, device=rowptr.device)
    call("dtc_tca_reorder", _ptr(rowptr), _ptr(col), num_nodes, col.numel(), C.byref(p),
         _ptr(perm), _ptr(ws), ws.numel(), _stream())
    return perm[:num_nodes]


def reorder(rowptr, col, val, num_nodes, params=None):
    """(perm, rowptr', col', val') with A' = P A Pᵀ under the TCA permutation."""
    perm = tca_perm(rowptr, col, num_nodes, params)
    rp, c, v = permute_csr(rowptr, col, val, perm)
    return perm, rp, c, v


def merge_pairs(sets, pairs, cap):
    """One level of the TCA greedy merge on given candidate pairs (dtc_tca_merge,
    host memory, no GPU): ``sets`` are the items' column sets, either a
    sequence of integer sequences or a tuple ``(ptr, idx)`` of CSR arrays
    whose rows are already sorted and distinct (the library checks); ``pairs``
    are (lo, hi) candidate pairs. Returns the root of every item (int32 numpy
    array)."""
    if isinstance(sets, tuple):
        ptr = np.ascontiguousarray(sets[0], np.int64)
        idx = np.ascontiguousarray(sets[1], np.int32)
        n = len(ptr) - 1
        if idx.size == 0:
            idx = np.zeros(1, np.int32)
    else:
        n = len(sets)
        norm = [np.unique(np.asarray(x, np.int64)) for x in sets]
        ptr = np.zeros(n + 1, np.int64)
        if n:
            ptr[1:] = np.cumsum([len(x) for x in norm])
        idx = (np.concatenate(norm) if n and ptr[-1] else np.zeros(1, np.int64)).astype(np.int32)
    pr = np.asarray(pairs, np.uint64).reshape(-1, 2)
    keys = np.ascontiguousarray((pr[:, 0] << np.uint64(32)) | pr[:, 1]) if len(pr) else \
        np.zeros(1, np.uint64)
    roots = np.zeros(max(n, 1), np.int32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    call("dtc_tca_merge", p(ptr), p(idx), n, p(keys), len(pr), int(cap), p(roots))
    return roots[:n]


def cluster_order(sets, candidates, thres=16, c_thres=128):
    """The two-level TCA clustering on a caller's candidate rule, host only:
    ``candidates(sets) -> [(lo, hi), ...]`` is called on the rows' column
    sets, then on the level-1 clusters' sets (the union of their rows' sets);
    each level merges with dtc_tca_merge (caps ``thres`` rows and ``c_thres``
    clusters). Returns perm[new] = old in the reference's output order
    (reordering/TCA_reorder.py:190-200, :296-307): level-2 groups by first
    appearance, their clusters ascending, each cluster's rows ascending. With
    the library's LSH as the rule this is what dtc_tca_reorder computes."""
    rows = [np.unique(np.asarray(x, np.int64)) for x in sets]

    def groups(roots):
        gid, out = {}, []
        for i, r in enumerate(roots.tolist()):
            if r not in gid:
                gid[r] = len(out)
                out.append([])
            out[gid[r]].append(i)
        return out
    g1 = groups(merge_pairs(rows, candidates(rows), thres))
    csets = [np.unique(np.concatenate([rows[i] for i in g])) for g in g1]
    g2 = groups(merge_pairs(csets, candidates(csets), c_thres))
    return np.array([r for g in g2 for c in g for r in g1[c]], np.int32)
