"""Many uneven sparse matrices (e.g. sampled GNN subgraphs) in one launch.

The matrices are stacked block-diagonally with each matrix's rows padded to a
whole number of 16-row windows, so no row window mixes two matrices and the
ME-TCF of the stack is exactly the union of the per-matrix ME-TCFs. One
conversion covers the whole batch, and one launch multiplies every matrix
with its own dense operand: the batch's TC blocks are cut into chunks
(contiguous block ranges, snapped to row windows in window mode) and one CTA
per SM pulls chunk ids from a device counter, the global work queue, until
the batch is done (queue=False runs one CTA per chunk instead, handed out by
the hardware block scheduler). The launch (plus its small chunk-table kernel
and, in balance mode, its partial-tile reduction) can be captured in a CUDA
graph and replayed.

There is no counterpart in the reference, which multiplies one matrix per
call (DTC-SpMM/DTCSpMM.cpp:117-178).
"""
from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import torch

from . import metcf as _m

WIN = 16


@dataclass
class BatchLayout:
    """Row offsets of each matrix inside the stacked (block-diagonal) matrix."""
    rows: np.ndarray        # int64 [B] rows of each matrix
    offsets: np.ndarray     # int64 [B+1] first stacked row of each matrix (multiples of 16)

    @property
    def total_rows(self):
        return int(self.offsets[-1])


def stack_csr(mats) -> (np.ndarray, np.ndarray, np.ndarray, BatchLayout):
    """Block-diagonal stack of square CSR matrices (objects with rowptr/col/val/M),
    each padded to a multiple of 16 rows with empty rows."""
    rows = np.array([m.M for m in mats], np.int64)
    padded = (rows + WIN - 1) // WIN * WIN
    offsets = np.zeros(len(mats) + 1, np.int64)
    offsets[1:] = np.cumsum(padded)
    total = int(offsets[-1])
    nnz = np.array([m.rowptr[-1] for m in mats], np.int64)
    if total >= 2 ** 31 or nnz.sum() >= 2 ** 31:
        raise ValueError("batch too large for int32 CSR indices")
    rowptr = np.zeros(total + 1, np.int64)
    col = np.empty(int(nnz.sum()), np.int32)
    val = np.empty(int(nnz.sum()), np.float32)
    e = 0
    for i, m in enumerate(mats):
        r0 = int(offsets[i])
        counts = np.diff(m.rowptr)
        rowptr[r0 + 1:r0 + 1 + m.M] = counts
        n = int(m.rowptr[-1])
        col[e:e + n] = m.col + r0
        val[e:e + n] = m.val
        e += n
    rowptr = np.cumsum(rowptr).astype(np.int32)
    return rowptr, col, val, BatchLayout(rows, offsets)


class BatchedSpMM:
    """C_i = A_i B_i for a list of square CSR matrices A_i, in one launch.

    `Bs` given to `run` is either a list of [rows_i x N] tensors (packed into
    the stacked operand on the device) or an already stacked [total_rows x N]
    tensor (rows of padding ignored). Results come back stacked; `split`
    returns per-matrix views.
    """

    def __init__(self, mats, N: int, device="cuda", fmt=None, precision=None, mode=1, grid=0,
                 queue=True):
        from ._lib import B_F32, PREC_TF32
        rowptr, col, val, self.layout = stack_csr(mats)
        self.N = N
        self.device = torch.device(device)
        self.fmt = B_F32 if fmt is None else fmt
        self.precision = PREC_TF32 if precision is None else precision
        self.mode, self.grid, self.ntile = mode, grid, 0
        self._csr = (rowptr, col, val)
        self.m = _m.convert(rowptr, col, self.layout.total_rows, values=val, device=self.device)
        self.B = torch.zeros((self.layout.total_rows, N), dtype=torch.float32, device=self.device)
        self.C = torch.empty((self.layout.total_rows, N), dtype=torch.float32, device=self.device)
        self.planes = None
        self.queue = queue
        self._alloc_ws()
        self.graph: Optional[torch.cuda.CUDAGraph] = None

    def _alloc_ws(self):
        """Workspace of the current schedule: partial tiles (balance mode) and,
        with queue=True, the chunk-queue region after them."""
        full = _m.spmm_ex_workspace_bytes(self.m, self.N, self.mode, self.grid)
        q = _m.spmm_ex_workspace_bytes(self.m, self.N, 0, self.grid)
        wsb = full if self.queue else full - q
        self.ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=self.device)

    def autotune(self, heights=(16, 32), reps=3):
        """Exhaustive schedule search for this batch (dtc_autotune): window height
        (16 or 32; a 32-row window may span two stacked matrices, which only adds
        distinct columns to it), strict balance or window mode, the CTA count
        (which sets the split threshold, blocks per CTA) and the N-tiles per CTA.
        Keeps the fastest and returns {height: best Schedule}."""
        from . import tune
        from ._lib import B_F32
        best, table = None, {}
        for h in heights:
            mm = self.m if h == self.m.H else _m.convert(*self._csr[:2], self.layout.total_rows,
                                                          H=h, values=self._csr[2],
                                                          device=self.device)
            planes = [self.B] if self.fmt == B_F32 else _m.pack_b(self.B, self.fmt)
            _, b = tune.autotune(mm, planes, self.fmt, self.N, self.precision, reps=reps,
                                 out=self.C)
            table[h] = b
            if best is None or b.ms < best[1].ms:
                best = (mm, b)
        self.m, sched = best
        self.mode, self.grid, self.ntile = sched.mode, sched.grid, sched.ntile
        self._alloc_ws()
        self.graph = None
        return table

    def load(self, Bs: List[torch.Tensor]):
        """Copy per-matrix operands into the stacked operand (rows beyond each
        matrix stay zero)."""
        off = self.layout.offsets
        for i, b in enumerate(Bs):
            self.B[int(off[i]):int(off[i]) + b.shape[0]].copy_(b, non_blocking=True)

    def _launch(self):
        from ._lib import B_F32
        if self.fmt == B_F32:
            planes = [self.B]
        else:  # storage planes allocated once, re-packed from the stacked operand every launch
            if self.planes is None:
                self.planes = _m.pack_b(self.B, self.fmt)
            planes = _m.pack_b_into(self.B, self.fmt, self.planes)
        _m.spmm_ex(self.m, planes, self.fmt, self.N, self.precision, mode=self.mode,
                   grid=self.grid, out=self.C, workspace=self.ws, ntile=self.ntile)

    def run(self):
        """One launch over the whole batch (graph replay when captured)."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self._launch()
        return self.C

    def capture(self, warmup=2):
        """Capture the batched SpMM in a CUDA graph (B changes between replays
        through `load`; the graph reads the stacked buffer in place)."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            for _ in range(warmup):
                self._launch()
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self._launch()
        self.graph = g
        return g

    def split(self, C=None):
        C = self.C if C is None else C
        off, rows = self.layout.offsets, self.layout.rows
        return [C[int(off[i]):int(off[i]) + int(rows[i])] for i in range(len(rows))]


def separate_launches(mats, N, device="cuda"):
    """The comparison point: one conversion and one window-scheduled launch per
    matrix (what a caller of the reference API does for a batch)."""
    ms = [_m.convert(a.rowptr, a.col, a.M, values=a.val, device=device) for a in mats]

    def run(Bs, outs):
        for mm, b, o in zip(ms, Bs, outs):
            _m.spmm(mm, b, out=o)
        return outs
    return ms, run


def separate_launches_graph(ms, Bs, outs, device="cuda"):
    """The per-matrix launches of separate_launches captured in ONE CUDA graph:
    the kernel-level baseline for the single batched launch (no host launch
    overhead between the matrices). Returns the graph; replay() reruns them."""
    s = torch.cuda.Stream(device)
    s.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(s):
        for mm, b, o in zip(ms, Bs, outs):
            _m.spmm(mm, b, out=o)
    torch.cuda.current_stream(device).wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for mm, b, o in zip(ms, Bs, outs):
            _m.spmm(mm, b, out=o)
    return g


def zipf_batch(count=512, N=64, seed=0, rows_lo=256, rows_hi=65536, s=2.1, dmin=1, dmax=2000):
    """The batched benchmark shape: `count` square matrices with log-uniform row
    counts in [rows_lo, rows_hi], Zipf(s) degrees truncated to [dmin, dmax],
    U(0,1) row-normalised values; dense operands rows x N of N(0,1)."""
    from . import gen
    rng = np.random.default_rng(seed)
    rows = np.exp(rng.uniform(np.log(rows_lo), np.log(rows_hi), count)).astype(np.int64)
    mats = [gen.zipf(int(r), s=s, dmin=dmin, dmax=min(dmax, int(r)), seed=seed * 100003 + i)
            for i, r in enumerate(rows)]
    Bs = [gen.normal(int(r), N, seed=seed * 7919 + i) for i, r in enumerate(rows)]
    return mats, Bs
