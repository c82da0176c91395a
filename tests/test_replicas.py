"""Multi-process (gloo, world size 2, CPU) tests of the multi-GPU plumbing:
row shards are window-aligned, cover the matrix and balance nonzeros; the
row-sharded product gathered on rank 0 equals the whole product; the timing
reduction takes the slowest rank."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from dtc_b200 import replicas


def test_shards_cover_and_balance():
    rng = np.random.default_rng(0)
    lens = rng.poisson(8, 1000)
    lens[37] = 3000  # a hub row
    rp = np.concatenate([[0], np.cumsum(lens)])
    for world in (1, 2, 3, 4):
        rs = [replicas.shard_rows(rp, world, r) for r in range(world)]
        assert rs[0][0] == 0 and rs[-1][1] == 1000
        assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
        assert all(r0 % 16 == 0 for r0, _ in rs)
        nz = [rp[r1] - rp[r0] for r0, r1 in rs]
        assert max(nz) <= rp[-1] / world + 3000 + 16 * 8 * 4


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from oracle import oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(1)
        M = 777
        rows = [np.sort(rng.choice(M, rng.integers(1, 12), replace=False)) for _ in range(M)]
        rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
        col = np.concatenate(rows).astype(np.int32)
        val = rng.standard_normal(len(col)).astype(np.float32)
        B = rng.standard_normal((M, 24)).astype(np.float32)
        r0, r1 = replicas.shard_rows(rp, world, rank)
        lrp, lcol, lval = replicas.sub_csr(rp, col, val, r0, r1)
        local = O.spmm_f64(lrp, lcol, lval, r1 - r0, B)
        C = replicas.gather_rows(local, dist)
        ms = replicas.max_over_ranks(1.0 + rank, dist)
        if rank == 0:
            full = O.spmm_f64(rp, col, val, M, B)
            q.put((bool(np.array_equal(C, full)), ms))
    finally:
        dist.destroy_process_group()


def test_row_sharded_product_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    equal, ms = q.get(timeout=10)
    assert equal
    assert ms == 2.0  # slowest of ranks' 1.0 and 2.0
    assert replicas.aggregate_gflops(1e9, 2.0, 2) == pytest.approx(1000.0)
