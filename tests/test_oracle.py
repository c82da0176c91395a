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


@pytest.mark.parametrize("path", _gpu_golden() or [None],
                         ids=lambda p: os.path.basename(p) if p else "none")
def test_oracle_matches_reference_gpu_preprocess(path):
    """Every block shape the reference was run with (16 x 8, 32 x 8, 16 x 16)."""
    if path is None:
        pytest.skip("no reference preprocess_gpu golden vectors present")
    name, H, W = cases.parse_golden_name(os.path.basename(path))
    g = np.load(path)
    rp, col, _, M = cases.CASES[name]()
    m = O.metcf(rp, col, M, H=H, W=W)
    assert m["T"] == int(g["T"])
    for k in ARRAYS:
        np.testing.assert_array_equal(m[k], g[k], err_msg=f"{name} {H}x{W}:{k}")


def test_gpu_golden_present_for_every_case_and_shape():
    found = {cases.parse_golden_name(os.path.basename(p)) for p in _gpu_golden()}
    if not found:
        pytest.skip("reference GPU golden vectors not generated yet")
    want = {(n, H, W) for n in cases.CASES for H, W in cases.GOLDEN_SHAPES}
    assert found == want, sorted(want - found)


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


@pytest.mark.parametrize("path", [p for p in _gpu_golden()
                                  if cases.parse_golden_name(os.path.basename(p))[1:] == (16, 8)]
                         or [None], ids=lambda p: os.path.basename(p) if p else "none")
def test_reference_spmm_golden_within_tf32_of_fp64(path):
    """The reference's own SpMM outputs (A = 1) are TF32 products of the FP64
    oracle's: N = 32 (float_nonsplit) and N = 128 (float4_split, stored rows)."""
    if path is None:
        pytest.skip("no reference golden vectors")
    from tests.golden import make_golden
    g = np.load(path)
    name = cases.parse_golden_name(os.path.basename(path))[0]
    rp, col, _, M = cases.CASES[name]()
    tol = 2.0 ** -9
    if "C_run" in g.files:
        bound = O.spmm_absbound_f64(rp, col, None, M, g["B"])
        c64 = O.spmm_f64(rp, col, None, M, g["B"])
        assert (np.abs(g["C_run"] - c64) <= tol * bound + 1e-6).all()
        assert (np.abs(g["C_balance"] / 1000.0 - c64) <= (tol + 1e-4) * bound + 1e-5).all()
    if "C_run128" in g.files:
        B = make_golden.b128(M)
        assert B.astype(np.float64).sum() == float(g["B128_sum"])
        rows = g["rows128"]
        bound = O.spmm_absbound_f64(rp, col, None, M, B)[rows]
        c64 = O.spmm_f64(rp, col, None, M, B)[rows]
        assert (np.abs(g["C_run128"] - c64) <= tol * bound + 1e-6).all()
        assert (np.abs(g["C_balance128"] / 1000.0 - c64) <= (tol + 1e-4) * bound + 1e-5).all()
