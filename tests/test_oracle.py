"""CPU tests: the oracle pinned against the reference's own outputs (golden
vectors in tests/golden/, produced by tests/golden/make_golden.py from the
unmodified reference), plus its internal consistency."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ARRAYS = ["RowWindowOffset", "TCblockRowid", "TCblocktileId", "TCblockoffset", "SparseAToX",
          "blockPartition", "edgeToColumn", "edgeToRow"]


@pytest.mark.parametrize("name", cases.CPU_REFERENCE_SAFE)
def test_oracle_matches_reference_cpu_preprocess(name):
    path = os.path.join(GOLDEN, f"ref_cpu_{name}.npz")
    g = np.load(path)
    rp, col, _, M = cases.CASES[name]()
    m = O.metcf(rp, col, M)
    # The CPU reference loops `iter < num_nodes + 1` (DTCSpMM.cpp:281): when
    # num_nodes % 16 == 0 it visits one window past the end, which has no
    # edges, and counts one extra block for it.
    assert m["T"] + (1 if M % 16 == 0 else 0) == int(g["T"])
    for k in ("blockPartition", "edgeToColumn", "edgeToRow"):
        np.testing.assert_array_equal(m[k], g[k], err_msg=k)


def _gpu_golden():
    return sorted(glob.glob(os.path.join(GOLDEN, "ref_gpu_*.npz")))


@pytest.mark.parametrize("path", _gpu_golden() or [None])
def test_oracle_matches_reference_gpu_preprocess(path):
    if path is None:
        pytest.skip("no reference preprocess_gpu golden vectors present")
    name = os.path.basename(path)[len("ref_gpu_"):-len(".npz")]
    g = np.load(path)
    rp, col, _, M = cases.CASES[name]()
    m = O.metcf(rp, col, M)
    assert m["T"] == int(g["T"])
    for k in ARRAYS:
        np.testing.assert_array_equal(m[k], g[k], err_msg=f"{name}:{k}")


def test_gpu_golden_present_for_every_case():
    names = {os.path.basename(p)[8:-4] for p in _gpu_golden()}
    if not names:
        pytest.skip("reference GPU golden vectors not generated yet")
    assert names == set(cases.CASES)


@pytest.mark.parametrize("name", list(cases.CASES))
def test_metcf_product_equals_csr_product(name):
    rp, col, val, M = cases.CASES[name]()
    m = O.metcf(rp, col, M, values=val)
    B = np.random.default_rng(7).standard_normal((M, 24)).astype(np.float32)
    # implicit A = 1: tile assignment collapses duplicate (row, col) pairs
    np.testing.assert_array_equal(O.metcf_spmm_f64(m, M, B), O.spmm_f64(rp, col, None, M, B))
    # real values: duplicates summed (fp32 sum in the tile array)
    np.testing.assert_allclose(O.metcf_spmm_f64(m, M, B, tc_values=m["TCvalues"]),
                               O.spmm_f64(rp, col, val, M, B), rtol=1e-5, atol=1e-5)


def test_all_ones_known_answer():
    # the reference's implied KAT (scripts/DTCSpMM/run_DTC_SpMM.py:68-76):
    # X = 1, A = 1  =>  C[i, :] = number of distinct columns of row i
    rp, col, _, M = cases.duplicates()
    B = np.ones((M, 8), np.float32)
    C = O.spmm_f64(rp, col, None, M, B)
    deg = np.array([len(set(col[rp[i]:rp[i + 1]])) for i in range(M)], np.float64)
    np.testing.assert_array_equal(C, np.repeat(deg[:, None], 8, axis=1))


def test_tile_values_merge_duplicates_first_occurrence():
    rp, col, val, M = cases.duplicates()
    m = O.metcf(rp, col, M, values=val)
    tv, tile, off = m["TCvalues"], m["TCblocktileId"], m["TCblockoffset"]
    for b in range(m["T"]):
        seen = set()
        for j in range(off[b], off[b + 1]):
            if tile[j] in seen:
                assert tv[j] == 0.0
            seen.add(tile[j])


def test_fp32_baseline_close_to_fp64():
    rp, col, val, M = cases.uniform_4096()
    B = np.random.default_rng(3).standard_normal((M, 32)).astype(np.float32)
    np.testing.assert_allclose(O.spmm_f32(rp, col, val, M, B, nthreads=2),
                               O.spmm_f64(rp, col, val, M, B), rtol=1e-4, atol=1e-5)
