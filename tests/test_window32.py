"""Row windows of height 32 (the autotuner's window-height knob): the
conversion with blockSize_h = 32 is bit-exact with the oracle (the reference
conversion takes blockSize_h as a parameter, DTC-SpMM/DTCSpMM.cpp:315-316),
and both kernel families compute the product within their tolerances for
every schedule, including windows split across CTAs and wide N."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import cases

pytestmark = pytest.mark.gpu


def _bound_ok(C, rp, col, val, M, B, tol):
    ref = O.spmm_f64(rp, col, val, M, B)
    bound = O.spmm_absbound_f64(rp, col, val, M, B)
    err = np.abs(C.astype(np.float64) - ref)
    ok = err <= tol * bound + 1e-6
    assert ok.all(), f"{(~ok).sum()} out of tolerance, worst {(err / (bound + 1e-30)).max():.3e}"


@pytest.mark.parametrize("name", ["small_uniform", "hub", "empty_windows", "duplicates",
                                  "banded_dense"])
def test_convert_h32_bit_exact(cuda, name):
    from dtc_b200 import metcf
    rp, col, val, M = cases.CASES[name]()
    m = metcf.convert(rp, col, M, H=32, values=val)
    ref = O.metcf(rp, col, M, H=32, values=val)
    assert m.T == ref["T"] and m.nwin == (M + 31) // 32
    for k in ("RowWindowOffset", "TCblockRowid", "TCblocktileId", "TCblockoffset", "SparseAToX",
              "TCvalues"):
        np.testing.assert_array_equal(getattr(m, k).cpu().numpy(), ref[k], err_msg=k)


@pytest.mark.parametrize("name", ["small_uniform", "hub", "empty_windows", "banded_dense"])
@pytest.mark.parametrize("form,N", [("tf32", 36), ("tf32", 128), ("tf32", 520),
                                    ("split24x4", 16), ("split24x4", 272), ("split24x3", 128),
                                    ("bf16x2x3", 128), ("bf16", 64), ("fp8", 32)])
@pytest.mark.parametrize("mode", [0, 1])
def test_spmm_h32(cuda, name, form, N, mode):
    import torch
    from dtc_b200 import metcf, tune
    rp, col, val, M = cases.CASES[name]()
    m = metcf.convert(rp, col, M, H=32, values=val)
    B = np.random.default_rng(21).standard_normal((M, N)).astype(np.float32)
    fmt, prec = tune.FORMS[form][0], tune.FORMS[form][1]
    Bd = torch.from_numpy(B).cuda()
    planes = [Bd] if form == "tf32" else metcf.pack_b(Bd, fmt)
    for grid in ((0, 5) if mode else (0,)):
        C = metcf.spmm_ex(m, planes, fmt, N, prec, mode=mode, grid=grid).cpu().numpy()
        if form == "tf32":
            _bound_ok(C, rp, col, val, M, B, 2.0 ** -9)
        elif form.startswith("split24") or form == "bf16x2x3":
            _bound_ok(C, rp, col, val, M, B, 2.0 ** -14)
        elif form == "bf16":
            _bound_ok(C, rp, col, val, M, B, 2.0 ** -8)
        else:
            _bound_ok(C, rp, col, val, M, (O.e4m3_values(O.pack_fp8(B)[0]) *
                                          O.pack_fp8(B)[1][:, None]).astype(np.float32), 2.0 ** -8)
    assert metcf.device_status(clear=True) == 0


@pytest.mark.parametrize("form,N", [("tf32", 512), ("split24x4", 512)])
def test_autotune_h32_all_schedules(cuda, form, N):
    import torch
    from dtc_b200 import gen, metcf, tune
    A = gen.zipf(5000, seed=8)
    m = metcf.convert(A.rowptr, A.col, A.M, H=32, values=A.val)
    B = gen.normal(A.M, N, seed=9)
    Bd = torch.from_numpy(B).cuda()
    fmt, prec = tune.FORMS[form][0], tune.FORMS[form][1]
    planes = [Bd] if form == "tf32" else metcf.pack_b(Bd, fmt)
    scheds, best = tune.autotune(m, planes, fmt, N, prec, reps=1)
    nts = {s.ntile for s in scheds}
    assert nts == ({1, 2, 4} if form == "tf32" else {1, 2})
    tol = 2.0 ** -9 if form == "tf32" else 2.0 ** -14
    for s in scheds:
        _bound_ok(tune.run(m, planes, fmt, N, prec, s).cpu().numpy(), A.rowptr, A.col, A.val,
                  A.M, B, tol)
    assert metcf.device_status(clear=True) == 0


def test_rejects_unsupported_height(cuda):
    import torch
    from dtc_b200 import metcf, DtcError
    rp, col, val, M = cases.small_uniform()
    m = metcf.convert(rp, col, M, H=8, values=val)
    with pytest.raises(DtcError, match="16 or 32"):
        metcf.spmm_ex(m, [torch.zeros((M, 16), device="cuda")], 0, 16, 0)


@pytest.mark.parametrize("name", ["small_uniform", "hub", "empty_windows", "banded_dense",
                                  "wide_window"])
@pytest.mark.parametrize("form,N", [("tf32", 36), ("tf32", 128), ("tf32", 520),
                                    ("split24x4", 16), ("split24x3", 272), ("bf16x2x3", 128),
                                    ("bf16", 64), ("fp8", 32)])
@pytest.mark.parametrize("mode", [0, 1])
def test_spmm_block_width_16(cuda, name, form, N, mode):
    """Compaction width 16 (blockSize_w = 16 at window height 16): every form
    and schedule on ME-TCF arrays of 16 x 16 blocks, within its tolerance."""
    import torch
    from dtc_b200 import metcf, tune
    rp, col, val, M = cases.CASES[name]()
    m = metcf.convert(rp, col, M, H=16, W=16, values=val)
    ref = O.metcf(rp, col, M, H=16, W=16, values=val)
    assert m.T == ref["T"]
    B = np.random.default_rng(22).standard_normal((M, N)).astype(np.float32)
    fmt, prec = tune.FORMS[form][0], tune.FORMS[form][1]
    Bd = torch.from_numpy(B).cuda()
    planes = [Bd] if form == "tf32" else metcf.pack_b(Bd, fmt)
    for grid in ((0, 5) if mode else (0,)):
        C = metcf.spmm_ex(m, planes, fmt, N, prec, mode=mode, grid=grid).cpu().numpy()
        if form == "tf32":
            _bound_ok(C, rp, col, val, M, B, 2.0 ** -9)
        elif form.startswith("split24") or form == "bf16x2x3":
            _bound_ok(C, rp, col, val, M, B, 2.0 ** -14)
        elif form == "bf16":
            _bound_ok(C, rp, col, val, M, B, 2.0 ** -8)
        else:
            _bound_ok(C, rp, col, val, M, (O.e4m3_values(O.pack_fp8(B)[0]) *
                                          O.pack_fp8(B)[1][:, None]).astype(np.float32), 2.0 ** -8)
    assert metcf.device_status(clear=True) == 0


def test_spmm_block_width_16_rejected_at_height_32(cuda):
    import torch
    from dtc_b200 import DtcError, metcf, B_F32, PREC_TF32
    rp, col, val, M = cases.hub()
    m = metcf.convert(rp, col, M, H=16, W=16, values=val)
    m.H = 32  # 32 x 16 tile ids would not fit a byte
    B = torch.zeros((M, 32), device="cuda")
    with pytest.raises(DtcError):
        metcf.spmm_ex(m, [B], B_F32, 32, PREC_TF32)
