"""Graph .npz loader (scripts/DTCSpMM/dataset.py:21-44): src_li / dst_li /
num_nodes -> CSR with every edge = 1 and duplicates summed, bit-exact with
scipy's coo -> csr (the reference's call), the oracle, and the reference
loader's own output (tests/golden/ref_loader_*.npz, made by
tests/golden/make_loader_golden.py)."""
import glob
import os

import numpy as np
import pytest

LOADER_GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden",
                                              "ref_loader_*.npz")))

from oracle import oracle as O


def _edges(n=500, m=6000, seed=0):
    rng = np.random.default_rng(seed)
    s = rng.integers(0, n, m)
    d = rng.integers(0, n, m)
    s[:40], d[:40] = s[40:80], d[40:80]  # duplicate edges
    return s, d, n


def test_oracle_coo_rebuild_matches_scipy():
    sp = pytest.importorskip("scipy.sparse")
    s, d, n = _edges()
    S = sp.coo_matrix((np.ones(len(s)), (s, d)), shape=(n, n)).tocsr()
    S.sum_duplicates()
    S.sort_indices()
    rp, c, v = O._coo_to_csr(s, d, None, n, n)
    np.testing.assert_array_equal(rp, S.indptr)
    np.testing.assert_array_equal(c, S.indices)
    np.testing.assert_array_equal(v, S.data.astype(np.float32))


def test_loader_golden_present():
    assert len(LOADER_GOLDEN) >= 3


@pytest.mark.parametrize("path", LOADER_GOLDEN, ids=lambda p: os.path.basename(p)[11:-4])
def test_oracle_matches_reference_loader(path):
    z = np.load(path)
    n = int(z["num_nodes"])
    rp, c, v = O._coo_to_csr(z["src_li"], z["dst_li"], None, n, n)
    np.testing.assert_array_equal(rp, z["row_pointers"])
    np.testing.assert_array_equal(c, z["column_index"])
    assert rp[-1] == rp[-2]  # the last node has no edges
    assert (v > 1).any()     # duplicate edges were summed


@pytest.mark.gpu
@pytest.mark.parametrize("path", LOADER_GOLDEN, ids=lambda p: os.path.basename(p)[11:-4])
def test_load_npz_matches_reference_loader(cuda, path):
    from dtc_b200 import dataset
    rp, col, val, n = dataset.load_npz(path)
    z = np.load(path)
    assert n == int(z["num_nodes"])
    np.testing.assert_array_equal(rp.cpu().numpy(), z["row_pointers"])
    np.testing.assert_array_equal(col.cpu().numpy(), z["column_index"])


@pytest.mark.gpu
def test_load_npz_bit_exact(cuda, tmp_path):
    from dtc_b200 import dataset
    s, d, n = _edges(seed=1)
    p = tmp_path / "g.npz"
    dataset.save_npz(p, s, d, n)
    rp, col, val, nn = dataset.load_npz(str(p))
    ref = O._coo_to_csr(s, d, None, n, n)
    assert nn == n
    np.testing.assert_array_equal(rp.cpu().numpy(), ref[0])
    np.testing.assert_array_equal(col.cpu().numpy(), ref[1])
    np.testing.assert_array_equal(val.cpu().numpy(), ref[2])


@pytest.mark.gpu
def test_coo_rejects_out_of_range(cuda):
    from dtc_b200 import dataset, DtcError
    with pytest.raises(DtcError, match="COO"):
        dataset.coo_to_csr(np.array([0, 5]), np.array([1, 1]), 4)
    rp, col, val = dataset.coo_to_csr(np.zeros(0, np.int32), np.zeros(0, np.int32), 3)
    np.testing.assert_array_equal(rp.cpu().numpy(), np.zeros(4, np.int32))
