"""Multi-GPU plumbing (one process per GPU, torch.distributed).

The path shards without any exchange: row windows are independent and the
strict balancer's partial tiles never leave a GPU. Two ways to use N GPUs:

* replicas (what ``bench.py --gpus N`` runs): every rank multiplies its own
  copy of the workload; throughput = all ranks' flops / the slowest rank's time;
* row shards: ``shard_rows`` cuts the rows at window boundaries into N ranges
  of near-equal nonzeros (the TC-block work follows the nonzeros); each rank
  converts and multiplies its own rows against a replicated B and keeps its C
  rows. No collective is on the data path; ``gather_rows`` is only for callers
  that want the whole C on one rank.
"""
import numpy as np


def shard_rows(rowptr, world, rank, H=16):
    """Row range [r0, r1) of `rank`: window-aligned, balanced by nonzeros."""
    rowptr = np.asarray(rowptr, np.int64)
    M = len(rowptr) - 1
    nwin = (M + H - 1) // H
    wend = np.minimum((np.arange(nwin + 1) * H), M)
    wnnz = rowptr[wend]  # nonzeros before each window boundary
    total = int(rowptr[-1])
    cuts = [0]
    for k in range(1, world):
        w = int(np.searchsorted(wnnz, total * k / world, side="left"))
        cuts.append(max(cuts[-1], min(w, nwin)))
    cuts.append(nwin)
    return int(wend[cuts[rank]]), int(wend[cuts[rank + 1]])


def sub_csr(rowptr, col, val, r0, r1):
    """Rows [r0, r1) of a CSR matrix (all columns kept)."""
    rowptr = np.asarray(rowptr)
    e0, e1 = int(rowptr[r0]), int(rowptr[r1])
    return ((rowptr[r0:r1 + 1] - e0).astype(np.int32), np.asarray(col)[e0:e1],
            None if val is None else np.asarray(val)[e0:e1])


def max_over_ranks(ms, dist=None, device=None):
    """Slowest rank's time (every rank must call this in the same order)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_gflops(flops_per_rank, ms_max, world):
    """Whole-job throughput of `world` replicas timed by their slowest rank."""
    return world * float(flops_per_rank) / (ms_max * 1e-3) / 1e9


def gather_rows(local_rows, dist, dst=0):
    """All ranks' C row blocks, in rank order, on rank `dst` (None elsewhere)."""
    out = [None] * dist.get_world_size() if dist.get_rank() == dst else None
    dist.gather_object(local_rows, out, dst=dst)
    return None if out is None else np.concatenate(out, axis=0)
