"""GPU tests of the dense-operand storage forms and the split-precision SpMM.

Packers are checked bit-exactly against the oracle's restatements. Each SpMM
form is checked twice: against the FP64 product with B *as stored* (tight:
only the A split and fp32 accumulation remain) and against the FP64 product
with the original fp32 B (the form's end-to-end accuracy).

Tolerances (per element, scaled by sum_e |a_e||b_e|):
  SPLIT24 (4-term or 3-term): stored-B 2^-15, original-B 2^-14
  BF16: stored-B 2^-15, original-B 2^-8
  FP8 (e4m3 + row scale): stored-B 2^-8 (q*scale is rounded to bf16), original-B 2^-3
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import cases

pytestmark = pytest.mark.gpu


def _u8(t):
    return t.cpu().numpy().view(np.uint8)


def _special_B(rows=64, N=48, seed=0):
    rng = np.random.default_rng(seed)
    B = (rng.standard_normal((rows, N)) * np.exp(rng.uniform(-20, 20, (rows, N)))).astype(np.float32)
    B[0, :8] = [0.0, -0.0, np.inf, -np.inf, np.nan, 1e-40, -1e-39, 3.4e38]
    B[1, :] = 0.0
    B[2, :4] = [1.0, 1.0 + 2 ** -16, 1.0 + 3 * 2 ** -16, -(1.0 + 2 ** -16)]  # RNE ties
    return B


def test_pack_split24_bit_exact(cuda):
    import torch
    from dtc_b200 import metcf, B_SPLIT24
    B = _special_B()
    hi, ext = O.pack_split24(B)
    p0, p1 = metcf.pack_b(torch.from_numpy(B).cuda(), B_SPLIT24)
    np.testing.assert_array_equal(_u8(p0).view(np.uint16).reshape(B.shape), hi)
    np.testing.assert_array_equal(_u8(p1).reshape(B.shape), ext)


def test_pack_bf16_bit_exact(cuda):
    import torch
    from dtc_b200 import metcf, B_BF16
    B = _special_B(seed=1)
    ref = O.pack_bf16(B)
    (p0,) = metcf.pack_b(torch.from_numpy(B).cuda(), B_BF16)
    got = _u8(p0).view(np.uint16).reshape(B.shape)
    nan = np.isnan(B)
    np.testing.assert_array_equal(got[~nan], ref[~nan])
    assert np.all((got[nan] & 0x7F80) == 0x7F80) and np.all(got[nan] & 0x7F)


def test_pack_fp8_bit_exact(cuda):
    import torch
    from dtc_b200 import metcf, B_FP8
    rng = np.random.default_rng(2)
    B = (rng.standard_normal((200, 64)) * np.exp(rng.uniform(-6, 6, (200, 1)))).astype(np.float32)
    B[3, :] = 0.0
    B[4, 5] = 1e-30  # deep subnormal after scaling
    q, s = O.pack_fp8(B)
    p0, p1 = metcf.pack_b(torch.from_numpy(B).cuda(), B_FP8)
    np.testing.assert_array_equal(_u8(p1).view(np.float32), s)
    np.testing.assert_array_equal(_u8(p0).reshape(B.shape), q)


def test_pack_bf16x2_bit_exact(cuda):
    import torch
    from dtc_b200 import metcf, B_BF16X2
    B = _special_B(seed=3)
    hi, lo = O.pack_bf16x2(B)
    p0, p1 = metcf.pack_b(torch.from_numpy(B).cuda(), B_BF16X2)
    gh = _u8(p0).view(np.uint16).reshape(B.shape)
    gl = _u8(p1).view(np.uint16).reshape(B.shape)
    ok = ~np.isnan(B)
    np.testing.assert_array_equal(gh[ok], hi[ok])
    np.testing.assert_array_equal(gl[ok], lo[ok])


def _stored_B(fmt, B):
    from dtc_b200 import B_BF16, B_BF16X2, B_FP8, B_SPLIT24
    if fmt == B_BF16X2:
        return O.bf16x2_values(*O.pack_bf16x2(B)).astype(np.float32)
    if fmt == B_SPLIT24:
        return O.split24_values(*O.pack_split24(B))
    if fmt == B_BF16:
        return (O.pack_bf16(B).astype(np.uint32) << 16).view(np.float32)
    if fmt == B_FP8:
        q, s = O.pack_fp8(B)
        return O.e4m3_values(q) * s[:, None]
    raise ValueError(fmt)


TOLS = {0: (2.0 ** -15, 2.0 ** -14), 1: (2.0 ** -15, 2.0 ** -14),   # SPLIT24 (by precision)
        "bf16": (2.0 ** -15, 2.0 ** -8), "fp8": (2.0 ** -8, 2.0 ** -3)}


def _run_form(name, N, fmt, prec, mode, grid=0):
    import torch
    from dtc_b200 import metcf
    rp, col, val, M = cases.CASES[name]()
    m = metcf.convert(rp, col, M, values=val)
    B = np.random.default_rng(5).standard_normal((M, N)).astype(np.float32)
    planes = metcf.pack_b(torch.from_numpy(B).cuda(), fmt)
    C = metcf.spmm_ex(m, planes, fmt, N, prec, mode=mode, grid=grid)
    return rp, col, val, M, B, C.cpu().numpy().astype(np.float64)


def _assert_close(C, rp, col, val, M, Bref, tol, what, abs_rows=None):
    """abs_rows: per-B-row absolute error allowance (e4m3 subnormal spacing)."""
    ref = O.spmm_f64(rp, col, val, M, Bref)
    bound = O.spmm_absbound_f64(rp, col, val, M, Bref)
    err = np.abs(C - ref)
    lim = tol * bound + 1e-6
    if abs_rows is not None:
        S = np.repeat(abs_rows.astype(np.float32)[:, None], Bref.shape[1], axis=1)
        lim = lim + O.spmm_absbound_f64(rp, col, val, M, S)
    assert (err <= lim).all(), f"{what}: {(err > lim).sum()} out of tolerance, worst {(err / (bound + 1e-30)).max():.3e}"


@pytest.mark.parametrize("name", ["small_uniform", "hub", "banded_dense", "empty_windows", "duplicates"])
@pytest.mark.parametrize("N", [16, 128, 272])
@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("mode", [0, 1])
def test_split24_forms(cuda, name, N, prec, mode):
    from dtc_b200 import B_SPLIT24
    rp, col, val, M, B, C = _run_form(name, N, B_SPLIT24, prec, mode)
    _assert_close(C, rp, col, val, M, _stored_B(B_SPLIT24, B), 2.0 ** -15, "stored B")
    _assert_close(C, rp, col, val, M, B, 2.0 ** -14, "original B")


@pytest.mark.parametrize("name", ["small_uniform", "hub", "banded_dense", "empty_windows"])
@pytest.mark.parametrize("N", [16, 128, 272])
@pytest.mark.parametrize("prec", [1, 2])
@pytest.mark.parametrize("mode", [0, 1])
def test_bf16x2_forms(cuda, name, N, prec, mode):
    from dtc_b200 import B_BF16X2
    rp, col, val, M, B, C = _run_form(name, N, B_BF16X2, prec, mode)
    _assert_close(C, rp, col, val, M, _stored_B(B_BF16X2, B), 2.0 ** -15, "stored B")
    _assert_close(C, rp, col, val, M, B, 2.0 ** -14, "original B")


@pytest.mark.parametrize("name", ["hub", "banded_dense"])
@pytest.mark.parametrize("N", [32, 256])
def test_bf16_and_fp8_forms(cuda, name, N):
    from dtc_b200 import B_BF16, B_FP8, PREC_SPLIT4
    for fmt, (t_stored, t_orig) in ((B_BF16, TOLS["bf16"]), (B_FP8, TOLS["fp8"])):
        for mode in (0, 1):
            rp, col, val, M, B, C = _run_form(name, N, fmt, PREC_SPLIT4, mode)
            _assert_close(C, rp, col, val, M, _stored_B(fmt, B), t_stored, f"fmt{fmt} stored")
            # e4m3 rounds to 2^-4 relative, or to 2^-10 * row scale in its subnormal range
            extra = O.pack_fp8(B)[1] * 2.0 ** -10 if fmt == B_FP8 else None
            _assert_close(C, rp, col, val, M, B, t_orig, f"fmt{fmt} original", abs_rows=extra)


@pytest.mark.parametrize("grid", [1, 5, 148])
def test_split_balance_deterministic(cuda, grid):
    from dtc_b200 import B_SPLIT24, PREC_SPLIT4
    a = _run_form("hub", 128, B_SPLIT24, PREC_SPLIT4, 1, grid)[-1]
    b = _run_form("hub", 128, B_SPLIT24, PREC_SPLIT4, 1, grid)[-1]
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_split_ones_known_answer(cuda):
    import torch
    from dtc_b200 import metcf, B_SPLIT24, PREC_SPLIT4
    rp, col, _, M = cases.duplicates()
    m = metcf.convert(rp, col, M)
    X = torch.ones((M, 16), device="cuda")
    planes = metcf.pack_b(X, B_SPLIT24)
    C = metcf.spmm_ex(m, planes, B_SPLIT24, 16, PREC_SPLIT4)
    deg = np.array([len(set(col[rp[i]:rp[i + 1]])) for i in range(M)], np.float32)
    np.testing.assert_array_equal(C.cpu().numpy(), np.repeat(deg[:, None], 16, axis=1))
    assert metcf.device_status(clear=True) == 0


def test_split_rejects_bad_shapes(cuda):
    import torch
    from dtc_b200 import metcf, B_SPLIT24, PREC_SPLIT4, PREC_TF32, DtcError
    rp, col, val, M = cases.small_uniform()
    m = metcf.convert(rp, col, M, values=val)
    B = torch.randn(M, 24, device="cuda")
    planes = metcf.pack_b(B, B_SPLIT24)
    with pytest.raises(DtcError):
        metcf.spmm_ex(m, planes, B_SPLIT24, 24, PREC_SPLIT4)   # N % 16 != 0
    with pytest.raises(DtcError):
        metcf.spmm_ex(m, planes, B_SPLIT24, 24, PREC_TF32)     # precision / format mismatch
