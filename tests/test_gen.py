"""CPU tests of the seeded synthetic generators (shapes and distributions of
the benchmark configurations)."""
import numpy as np

from dtc_b200 import gen


def _check_csr(m, square=True):
    assert m.rowptr[0] == 0 and np.all(np.diff(m.rowptr) >= 0)
    assert m.rowptr[-1] == len(m.col) == len(m.val)
    assert m.col.min() >= 0 and m.col.max() < m.K
    for i in range(0, m.M, max(1, m.M // 50)):
        r = m.col[m.rowptr[i]:m.rowptr[i + 1]]
        assert np.all(np.diff(r) > 0)  # sorted, no duplicates


def test_uniform_small_config_shape():
    m = gen.uniform(4096, mean=8.0, seed=0)
    _check_csr(m)
    assert abs(m.nnz - 4096 * 8) < 4 * np.sqrt(4096 * 8)
    assert m.val.min() >= -1 and m.val.max() <= 1


def test_deterministic():
    a = gen.uniform(1000, mean=5, seed=3)
    b = gen.uniform(1000, mean=5, seed=3)
    c = gen.uniform(1000, mean=5, seed=4)
    np.testing.assert_array_equal(a.col, b.col)
    np.testing.assert_array_equal(a.val, b.val)
    assert not np.array_equal(a.col[:100], c.col[:100])
    np.testing.assert_array_equal(gen.normal(10, 7, seed=1), gen.normal(10, 7, seed=1))


def test_rmat_symmetric_selfloops_gcn():
    m = gen.rmat(scale=10, edge_factor=16, seed=0)
    _check_csr(m)
    import scipy.sparse as sp
    A = sp.csr_matrix((m.val, m.col, m.rowptr), shape=(m.M, m.M))
    assert abs(A - A.T).max() < 1e-6
    assert np.all(A.diagonal() > 0)
    deg = np.diff(m.rowptr).astype(np.float64)
    i = 5
    e = m.rowptr[i]
    assert np.isclose(m.val[e], 1 / np.sqrt(deg[i] * deg[m.col[e]]), rtol=1e-6)


def test_stencil27_counts_and_diagonal():
    n = 10
    m = gen.stencil27(n, seed=0)
    _check_csr(m)
    assert m.M == n ** 3 and m.nnz == (3 * n - 2) ** 3
    i = 555
    r = slice(m.rowptr[i], m.rowptr[i + 1])
    cols, vals = m.col[r], m.val[r]
    d = vals[cols == i][0]
    assert np.isclose(d, 27 + abs(vals[cols != i].astype(np.float64).sum()), rtol=1e-5)


def test_zipf_degrees_and_row_normalised():
    m = gen.zipf(5000, s=2.1, dmin=1, dmax=2000, seed=1)
    _check_csr(m)
    deg = np.diff(m.rowptr)
    assert deg.min() >= 1 and deg.max() <= 2000
    sums = np.add.reduceat(m.val.astype(np.float64), m.rowptr[:-1])
    np.testing.assert_allclose(sums, 1.0, rtol=1e-5)


def test_structured_families():
    _check_csr(gen.banded(2000, 16, 0.5, seed=0))
    _check_csr(gen.blockdiag(2000, 64, 12, 0.05, seed=0))
