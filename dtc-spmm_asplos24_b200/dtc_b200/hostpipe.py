"""C = A·B for dense operands that live in host memory, copies overlapped.

A GNN layer whose features sit on the host (a feature store, a data loader)
pays two PCIe copies per product: B in (rows x N fp32) and C out, each far
longer than the SpMM itself. ``HostPipeline`` runs them on three CUDA streams

    copy-in : pinned host B  -> device B buffer (i % 2)
    compute : [row gather by the reorder permutation] -> pack into the B
              storage form -> SpMM (the tuned schedule) -> device C buffer (i % 2)
    copy-out: device C buffer (i % 2) -> pinned host C

with two device buffers each for B and C, so product i+1's B copy runs
while product i computes and copies its C out (PCIe moves both directions at
once). Every buffer is allocated up front; ``submit`` enqueues one product
and returns. The reference has no host-side path: its API takes and returns
device tensors (DTC-SpMM/DTCSpMM.cpp:117-178).
"""
import torch

from . import metcf
from .metcf import METCF


class HostPipeline:
    """Streams products C_i = A · B_i for host-resident B_i / C_i.

    m         ME-TCF of A (device)
    N         columns of B and C
    fmt, precision, mode, grid, ntile
              the storage form and schedule of the SpMM (as in metcf.spmm_ex)
    perm      optional device permutation (new -> old) when A was reordered:
              row i of the product's B is row perm[i] of the caller's B
    """

    def __init__(self, m: METCF, N, fmt, precision, mode=0, grid=0, ntile=0, perm=None,
                 use_values=True):
        dev = m.RowWindowOffset.device
        self.m, self.N, self.fmt, self.precision = m, N, fmt, precision
        self.mode, self.grid, self.ntile, self.use_values = mode, grid, ntile, use_values
        self.perm = None if perm is None else perm.to(device=dev, dtype=torch.long)
        f32 = dict(dtype=torch.float32, device=dev)
        self.B = [torch.empty((m.M, N), **f32) for _ in range(2)]
        self.C = [torch.empty((m.M, N), **f32) for _ in range(2)]
        self.Bp = torch.empty((m.M, N), **f32) if perm is not None else None
        self.planes = None if fmt == 0 else metcf.pack_b(self.B[0], fmt)
        wsb = metcf.spmm_ex_workspace_bytes(m, N, mode, grid)
        self.ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=dev)
        self.s_in = torch.cuda.Stream(device=dev)
        self.s_comp = torch.cuda.Stream(device=dev)
        self.s_out = torch.cuda.Stream(device=dev)
        self.ev_in = [torch.cuda.Event() for _ in range(2)]     # B buffer filled
        self.ev_free = [torch.cuda.Event() for _ in range(2)]   # B buffer consumed
        self.ev_comp = [torch.cuda.Event() for _ in range(2)]   # C buffer written
        self.ev_out = [torch.cuda.Event() for _ in range(2)]    # C buffer copied out
        self.i = 0
        self.launches_per_product = metcf.spmm_ex_launches(m, mode, grid) + \
            (0 if fmt == 0 else 1)

    def submit(self, B_host, C_host):
        """Enqueues C_host = A · B_host (both pinned fp32 [M, N] host tensors)."""
        k = self.i & 1
        if self.i >= 2:
            self.s_in.wait_event(self.ev_free[k])
        with torch.cuda.stream(self.s_in):
            self.B[k].copy_(B_host, non_blocking=True)
            self.ev_in[k].record(self.s_in)
        self.s_comp.wait_event(self.ev_in[k])
        with torch.cuda.stream(self.s_comp):
            Bk = self.B[k]
            if self.perm is not None:
                torch.index_select(Bk, 0, self.perm, out=self.Bp)
                Bk = self.Bp
            planes = [Bk] if self.fmt == 0 else metcf.pack_b_into(Bk, self.fmt, self.planes)
            self.ev_free[k].record(self.s_comp)
            if self.i >= 2:
                self.s_comp.wait_event(self.ev_out[k])
            metcf.spmm_ex(self.m, planes, self.fmt, self.N, self.precision, mode=self.mode,
                          grid=self.grid, ntile=self.ntile, use_values=self.use_values,
                          out=self.C[k], workspace=self.ws)
            self.ev_comp[k].record(self.s_comp)
        self.s_out.wait_event(self.ev_comp[k])
        with torch.cuda.stream(self.s_out):
            C_host.copy_(self.C[k], non_blocking=True)
            self.ev_out[k].record(self.s_out)
        self.i += 1

    @property
    def streams(self):
        return self.s_in, self.s_comp, self.s_out

    def synchronize(self):
        for s in self.streams:
            s.synchronize()
