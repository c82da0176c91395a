"""CSR relabelling: applying a reorder permutation (reordering/TCA_reorder.py
:308-326 + the scipy CSR rebuild of scripts/DTCSpMM/dataset.py:38-44) and
transposition.

CPU: the oracle's restatement is pinned against scipy's coo -> csr, the call
the reference makes. GPU: dtc_permute_csr / dtc_transpose_csr are bit-exact
with the oracle (row pointer, columns, summed values), and ME-TCF conversion of
the permuted matrix is bit-exact with the oracle conversion of the oracle's
permuted matrix.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import cases


def _coo_case(M=257, nnz=4000, seed=0, dup=True):
    rng = np.random.default_rng(seed)
    r = rng.integers(0, M, nnz)
    c = rng.integers(0, M, nnz)
    if dup:
        r[:50], c[:50] = r[50:100], c[50:100]  # guaranteed duplicates
    r[r == 7] = 8  # an empty row
    v = rng.standard_normal(nnz).astype(np.float32)
    o = np.argsort(r, kind="stable")
    rp = np.zeros(M + 1, np.int64)
    np.add.at(rp, r + 1, 1)
    return np.cumsum(rp).astype(np.int32), c[o].astype(np.int32), v[o], M


def _scipy_canonical(rows, r, c, v, shape):
    sp = pytest.importorskip("scipy.sparse")
    S = sp.coo_matrix((v, (r, c)), shape=shape).tocsr()
    S.sum_duplicates()
    S.sort_indices()
    return S


@pytest.mark.parametrize("seed", [0, 1])
def test_oracle_permute_matches_scipy_rebuild(seed):
    rp, col, val, M = _coo_case(seed=seed)
    perm = np.random.default_rng(seed + 10).permutation(M)
    d = np.empty(M, np.int64)
    d[perm] = np.arange(M)
    src = np.repeat(np.arange(M), np.diff(rp))
    ones = np.ones(len(col), np.float32)  # the reference's A = 1: duplicates count
    S = _scipy_canonical(M, d[src], d[col], ones, (M, M))
    orp, oc, ov = O.permute_csr(rp, col, None, perm)
    np.testing.assert_array_equal(orp, S.indptr)
    np.testing.assert_array_equal(oc, S.indices)
    np.testing.assert_array_equal(ov, S.data.astype(np.float32))
    assert ov.max() >= 2.0  # duplicates were merged


def test_oracle_transpose_matches_scipy():
    rp, col, val, M = _coo_case(seed=3, dup=False)
    src = np.repeat(np.arange(M), np.diff(rp))
    S = _scipy_canonical(M, col, src, val, (M, M))
    orp, oc, ov = O.transpose_csr(rp, col, val, M)
    np.testing.assert_array_equal(orp, S.indptr)
    np.testing.assert_array_equal(oc, S.indices)
    np.testing.assert_allclose(ov, S.data, rtol=0, atol=0)


def test_oracle_rejects_non_permutation():
    rp, col, val, M = _coo_case()
    with pytest.raises(ValueError):
        O.permute_csr(rp, col, val, np.zeros(M, np.int64))


def _gpu(x, dtype=None):
    import torch
    return torch.as_tensor(np.asarray(x) if dtype is None else np.asarray(x, dtype)).cuda()


def _np(t):
    return t.cpu().numpy()


@pytest.mark.gpu
@pytest.mark.parametrize("with_values", [True, False])
@pytest.mark.parametrize("seed", [0, 1, 2])
def test_permute_bit_exact(cuda, seed, with_values):
    from dtc_b200 import metcf
    rp, col, val, M = _coo_case(seed=seed)
    perm = np.random.default_rng(seed + 10).permutation(M).astype(np.int32)
    v = val if with_values else None
    grp, gc, gv = metcf.permute_csr(_gpu(rp), _gpu(col), None if v is None else _gpu(v),
                                    _gpu(perm))
    orp, oc, ov = O.permute_csr(rp, col, v, perm)
    np.testing.assert_array_equal(_np(grp), orp)
    np.testing.assert_array_equal(_np(gc), oc)
    np.testing.assert_array_equal(_np(gv).view(np.uint32), ov.view(np.uint32))


@pytest.mark.gpu
def test_transpose_bit_exact_rectangular(cuda):
    from dtc_b200 import metcf
    rng = np.random.default_rng(4)
    M, K = 100, 333
    rows = [np.sort(rng.choice(K, rng.integers(0, 20), replace=False)) for _ in range(M)]
    rp = np.concatenate([[0], np.cumsum([len(x) for x in rows])]).astype(np.int32)
    col = np.concatenate(rows).astype(np.int32)
    val = rng.standard_normal(len(col)).astype(np.float32)
    grp, gc, gv = metcf.transpose_csr(_gpu(rp), _gpu(col), _gpu(val), K)
    orp, oc, ov = O.transpose_csr(rp, col, val, K)
    assert len(orp) == K + 1
    np.testing.assert_array_equal(_np(grp), orp)
    np.testing.assert_array_equal(_np(gc), oc)
    np.testing.assert_array_equal(_np(gv), ov)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["small_uniform", "hub", "empty_windows", "duplicates"])
def test_permuted_metcf_bit_exact(cuda, name):
    """Reorder then convert: the ME-TCF arrays of P A Pᵀ equal the oracle's."""
    from dtc_b200 import metcf
    rp, col, val, M = cases.CASES[name]()
    perm = np.random.default_rng(7).permutation(M).astype(np.int32)
    grp, gc, gv = metcf.permute_csr(_gpu(rp), _gpu(col), _gpu(val), _gpu(perm))
    m = metcf.convert(grp, gc, M, values=gv)
    orp, oc, ov = O.permute_csr(rp, col, val, perm)
    ref = O.metcf(orp, oc, M)
    np.testing.assert_array_equal(_np(m.RowWindowOffset), ref["RowWindowOffset"])
    np.testing.assert_array_equal(_np(m.TCblocktileId), ref["TCblocktileId"])
    np.testing.assert_array_equal(_np(m.TCblockoffset), ref["TCblockoffset"])
    np.testing.assert_array_equal(_np(m.SparseAToX), ref["SparseAToX"])


@pytest.mark.gpu
def test_transposed_spmm_matches_fp64(cuda):
    """Aᵀ·G through transpose + conversion + TF32 SpMM (the true backward product)."""
    import torch
    from dtc_b200 import metcf
    rp, col, val, M = cases.hub()
    trp, tc, tv = metcf.transpose_csr(_gpu(rp), _gpu(col), _gpu(val), M)
    m = metcf.convert(trp, tc, M, values=tv)
    G = np.random.default_rng(9).standard_normal((M, 64)).astype(np.float32)
    C = metcf.spmm(m, torch.from_numpy(G).cuda()).cpu().numpy().astype(np.float64)
    orp, oc, ov = O.transpose_csr(rp, col, val, M)
    ref = O.spmm_f64(orp, oc, ov, M, G)
    bound = O.spmm_absbound_f64(orp, oc, ov, M, G)
    assert (np.abs(C - ref) <= 2.0 ** -9 * bound + 1e-6).all()


@pytest.mark.gpu
def test_relabel_rejects_bad_inputs(cuda):
    from dtc_b200 import metcf, DtcError
    rp, col, val, M = _coo_case()
    bad_perm = np.arange(M, dtype=np.int32)
    bad_perm[3] = bad_perm[4]
    with pytest.raises(DtcError, match="permutation"):
        metcf.permute_csr(_gpu(rp), _gpu(col), None, _gpu(bad_perm))
    bad_col = col.copy()
    bad_col[5] = M + 3
    with pytest.raises(DtcError, match="invalid CSR"):
        metcf.permute_csr(_gpu(rp), _gpu(bad_col), None, _gpu(np.arange(M, dtype=np.int32)))
    empty = metcf.permute_csr(_gpu(np.zeros(5, np.int32)), _gpu(np.zeros(0, np.int32)), None,
                              _gpu(np.arange(4, dtype=np.int32)))
    np.testing.assert_array_equal(_np(empty[0]), np.zeros(5, np.int32))
    assert empty[1].numel() == 0
