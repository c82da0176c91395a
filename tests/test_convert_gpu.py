"""GPU parity of the ME-TCF conversion (through the C ABI): bit-exact with the
oracle and with the reference's own preprocess_gpu golden vectors."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import cases

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
ARRAYS = ["RowWindowOffset", "TCblockRowid", "TCblocktileId", "TCblockoffset", "SparseAToX",
          "blockPartition", "edgeToColumn", "edgeToRow"]


def _gpu_convert(rp, col, M, val=None, H=16, W=8):
    from dtc_b200 import metcf
    m = metcf.convert(rp, col, M, H=H, W=W, values=val)
    out = {k: getattr(m, k).cpu().numpy() for k in ARRAYS}
    out["T"] = m.T
    if val is not None:
        out["TCvalues"] = m.TCvalues.cpu().numpy()
    return out


def _assert_same(got, exp, tag):
    assert got["T"] == exp["T"], tag
    for k in ARRAYS:
        np.testing.assert_array_equal(got[k], exp[k], err_msg=f"{tag}:{k}")


@pytest.mark.parametrize("name", list(cases.CASES))
def test_convert_bit_exact_vs_oracle(cuda, name):
    rp, col, val, M = cases.CASES[name]()
    got = _gpu_convert(rp, col, M, val)
    exp = O.metcf(rp, col, M, values=val)
    _assert_same(got, exp, name)
    np.testing.assert_array_equal(got["TCvalues"], exp["TCvalues"])


@pytest.mark.parametrize("name", list(cases.CASES))
@pytest.mark.parametrize("hw", cases.GOLDEN_SHAPES, ids=lambda hw: f"{hw[0]}x{hw[1]}")
def test_convert_bit_exact_vs_reference_golden(cuda, name, hw):
    H, W = hw
    path = os.path.join(GOLDEN, cases.golden_name(name, H, W))
    if not os.path.exists(path):
        pytest.skip("reference golden vector not generated")
    g = dict(np.load(path))
    g["T"] = int(g["T"])
    rp, col, _, M = cases.CASES[name]()
    _assert_same(_gpu_convert(rp, col, M, H=H, W=W), g, f"{name} {H}x{W}")


@pytest.mark.parametrize("hw", [(16, 8), (16, 16), (32, 8), (8, 8)])
def test_convert_other_block_shapes(cuda, hw):
    H, W = hw
    rp, col, val, M = cases.wide_window()
    got = _gpu_convert(rp, col, M, val, H=H, W=W)
    exp = O.metcf(rp, col, M, H=H, W=W, values=val)
    _assert_same(got, exp, f"{H}x{W}")


def test_convert_generated_configs(cuda):
    from dtc_b200 import gen
    for m in (gen.uniform(4096, mean=8, seed=0), gen.rmat(scale=14, seed=2),
              gen.stencil27(20, seed=0), gen.zipf(20000, seed=3)):
        got = _gpu_convert(m.rowptr, m.col, m.M, m.val)
        exp = O.metcf(m.rowptr, m.col, m.M, values=m.val)
        _assert_same(got, exp, "generated")
        np.testing.assert_array_equal(got["TCvalues"], exp["TCvalues"])


def _full_size(name):
    from dtc_b200 import gen
    if name == "uniform_4096":
        return gen.uniform(4096, mean=8.0, seed=0)
    if name == "rmat20":
        return gen.rmat(20, 16.0, 0.57, 0.19, 0.19, seed=0)
    return gen.stencil27(126, seed=0)


@pytest.mark.parametrize("name,H,W", [("uniform_4096", 16, 8), ("rmat20", 16, 8),
                                      ("rmat20", 32, 8), ("rmat20", 16, 16),
                                      ("stencil126", 16, 8), ("stencil126", 32, 8)])
def test_convert_full_size_configs(cuda, name, H, W):
    """Every ME-TCF array at the benchmark sizes, bit-exact with the oracle:
    uniform 4096^2 Poisson(8), R-MAT 2^20 symmetrised + I (32.5 M nnz, hub
    windows of ~15k TC blocks) and the 27-point stencil on 126^3 (2,000,376
    rows, num_nodes % 16 == 8)."""
    A = _full_size(name)
    got = _gpu_convert(A.rowptr, A.col, A.M, A.val, H=H, W=W)
    exp = O.metcf(A.rowptr, A.col, A.M, H=H, W=W, values=A.val)
    _assert_same(got, exp, f"{name} {H}x{W}")
    np.testing.assert_array_equal(got["TCvalues"], exp["TCvalues"])


def test_convert_empty_matrix(cuda):
    M = 50
    rp = np.zeros(M + 1, np.int32)
    got = _gpu_convert(rp, np.zeros(0, np.int32), M)
    assert got["T"] == 0
    assert np.all(got["RowWindowOffset"] == 0)


def test_convert_rejects_invalid_csr(cuda):
    from dtc_b200 import DtcError
    rp, col, _, M = cases.small_uniform()
    bad = col.copy()
    bad[3] = M + 5
    with pytest.raises(DtcError):
        _gpu_convert(rp, bad, M)
    rp2 = rp.copy()
    rp2[10] = rp2[11] + 1
    with pytest.raises(DtcError):
        _gpu_convert(rp2, col, M)


def test_extension_preprocess_gpu_matches(cuda):
    import torch
    import DTCSpMM
    rp, col, val, M = cases.hub()
    nwin = (M + 15) // 16
    dev = torch.device("cuda")
    bp = torch.zeros(nwin, dtype=torch.int32, device=dev)
    e2c = torch.zeros(len(col), dtype=torch.int32, device=dev)
    e2r = torch.zeros(len(col), dtype=torch.int32, device=dev)
    res = DTCSpMM.preprocess_gpu(torch.from_numpy(col).to(dev), torch.from_numpy(rp).to(dev), M,
                                 16, 8, bp, e2c, e2r)
    exp = O.metcf(rp, col, M)
    names = ["RowWindowOffset", "TCblockRowid", "TCblocktileId", "TCblockoffset", "SparseAToX"]
    for k, t in zip(names, res[:5]):
        np.testing.assert_array_equal(t.cpu().numpy(), exp[k], err_msg=k)
    assert res[5] == exp["T"]
    np.testing.assert_array_equal(bp.cpu().numpy(), exp["blockPartition"])
    np.testing.assert_array_equal(e2c.cpu().numpy(), exp["edgeToColumn"])
    np.testing.assert_array_equal(e2r.cpu().numpy(), exp["edgeToRow"])
    res_v = DTCSpMM.preprocess_gpu(torch.from_numpy(col).to(dev), torch.from_numpy(rp).to(dev),
                                   M, 16, 8, bp, e2c, e2r, values=torch.from_numpy(val).to(dev))
    assert len(res_v) == 7
    exp_v = O.metcf(rp, col, M, values=val)
    np.testing.assert_array_equal(res_v[6].cpu().numpy(), exp_v["TCvalues"])
