"""Batched SpMM: block-diagonal stacking (CPU) and one-launch / graph-replay
results against the FP64 oracle (GPU)."""
import numpy as np
import pytest

from dtc_b200 import batched, gen
from oracle import oracle as O

TF32_TOL = 2.0 ** -9


def _mats(count=12, seed=3):
    rng = np.random.default_rng(seed)
    return [gen.zipf(int(r), s=2.1, dmin=1, dmax=min(200, int(r)), seed=seed * 1000 + i)
            for i, r in enumerate(rng.integers(5, 700, count))]


def test_stack_layout_and_block_diagonal():
    mats = _mats()
    rp, col, val, lay = batched.stack_csr(mats)
    assert lay.offsets[0] == 0 and np.all(lay.offsets % 16 == 0)
    assert np.all(np.diff(lay.offsets) >= lay.rows)
    assert rp[-1] == sum(m.nnz for m in mats)
    for i, m in enumerate(mats):
        r0 = int(lay.offsets[i])
        seg = slice(rp[r0], rp[r0 + m.M])
        np.testing.assert_array_equal(col[seg] - r0, m.col)
        np.testing.assert_array_equal(val[seg], m.val)
        # padding rows are empty
        assert rp[r0 + m.M] == rp[int(lay.offsets[i + 1])]
    # ME-TCF of the stack = union of per-matrix ME-TCFs (windows never mix matrices)
    whole = O.metcf(rp, col, lay.total_rows)
    assert whole["T"] == sum(O.metcf(m.rowptr, m.col, m.M)["T"] for m in mats)


def test_zipf_batch_shapes():
    mats, Bs = batched.zipf_batch(count=8, N=16, seed=1, rows_lo=256, rows_hi=4096)
    assert len(mats) == 8 and all(256 <= m.M <= 4096 for m in mats)
    assert all(b.shape == (m.M, 16) for m, b in zip(mats, Bs))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
def test_batched_matches_oracle_and_graph_replay(cuda, mode):
    import torch
    mats = _mats(20)
    N = 64
    rng = np.random.default_rng(0)
    Bs = [rng.standard_normal((m.M, N)).astype(np.float32) for m in mats]
    bs = batched.BatchedSpMM(mats, N, mode=mode)
    bs.load([torch.from_numpy(b).cuda() for b in Bs])
    outs = [c.cpu().numpy() for c in bs.split(bs.run())]
    for m, b, c in zip(mats, Bs, outs):
        ref = O.spmm_f64(m.rowptr, m.col, m.val, m.M, b)
        bound = O.spmm_absbound_f64(m.rowptr, m.col, m.val, m.M, b)
        assert (np.abs(c - ref) <= TF32_TOL * bound + 1e-6).all()
    # graph capture, then replay with new operands
    bs.capture()
    Bs2 = [rng.standard_normal((m.M, N)).astype(np.float32) for m in mats]
    bs.load([torch.from_numpy(b).cuda() for b in Bs2])
    outs2 = [c.cpu().numpy() for c in bs.split(bs.run())]
    for m, b, c in zip(mats, Bs2, outs2):
        ref = O.spmm_f64(m.rowptr, m.col, m.val, m.M, b)
        bound = O.spmm_absbound_f64(m.rowptr, m.col, m.val, m.M, b)
        assert (np.abs(c - ref) <= TF32_TOL * bound + 1e-6).all()


@pytest.mark.gpu
def test_batched_split_form_in_graph(cuda):
    import torch
    from dtc_b200 import B_SPLIT24, PREC_SPLIT4
    mats = _mats(10, seed=5)
    N = 32
    rng = np.random.default_rng(2)
    bs = batched.BatchedSpMM(mats, N, fmt=B_SPLIT24, precision=PREC_SPLIT4)
    bs.capture()
    Bs = [rng.standard_normal((m.M, N)).astype(np.float32) for m in mats]
    bs.load([torch.from_numpy(b).cuda() for b in Bs])
    for m, b, c in zip(mats, Bs, [c.cpu().numpy() for c in bs.split(bs.run())]):
        ref = O.spmm_f64(m.rowptr, m.col, m.val, m.M, b)
        bound = O.spmm_absbound_f64(m.rowptr, m.col, m.val, m.M, b)
        assert (np.abs(c - ref) <= 2.0 ** -14 * bound + 1e-6).all()


@pytest.mark.gpu
def test_batched_autotune_then_graph(cuda):
    """The autotuner's pick (window height, mode, CTA count, N-tiles) for the
    batch keeps every matrix's product correct, also under graph replay."""
    import torch
    mats = _mats(16, seed=7)
    N = 64
    rng = np.random.default_rng(4)
    bs = batched.BatchedSpMM(mats, N)
    table = bs.autotune(reps=1)
    assert set(table) == {16, 32} and bs.m.H in (16, 32)
    bs.capture()
    Bs = [rng.standard_normal((m.M, N)).astype(np.float32) for m in mats]
    bs.load([torch.from_numpy(b).cuda() for b in Bs])
    for m, b, c in zip(mats, Bs, [c.cpu().numpy() for c in bs.split(bs.run())]):
        ref = O.spmm_f64(m.rowptr, m.col, m.val, m.M, b)
        bound = O.spmm_absbound_f64(m.rowptr, m.col, m.val, m.M, b)
        assert (np.abs(c - ref) <= TF32_TOL * bound + 1e-6).all()
