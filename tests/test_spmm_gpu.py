"""GPU parity of the TC-block SpMM kernels (through the C ABI) against the
FP64 oracle, the reference's own SpMM golden outputs and the all-ones KAT.

Tolerance (TF32 form): |C - C64| <= 2^-9 * sum_e |a_e| |b_e| + 1e-6 per
element: A is rounded to TF32 (2^-11), B is read by the tensor core at TF32
precision (truncation, 2^-10), products accumulate in fp32.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import cases

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TF32_TOL = 2.0 ** -9


def _setup(name, N, seed=11):
    import torch
    from dtc_b200 import metcf
    rp, col, val, M = cases.CASES[name]()
    m = metcf.convert(rp, col, M, values=val)
    B = np.random.default_rng(seed).standard_normal((M, N)).astype(np.float32)
    return rp, col, val, M, m, B, torch.from_numpy(B).cuda()


def _check(C, rp, col, val, M, B, tol=TF32_TOL):
    C = C.cpu().numpy().astype(np.float64)
    ref = O.spmm_f64(rp, col, val, M, B)
    bound = O.spmm_absbound_f64(rp, col, val, M, B)
    err = np.abs(C - ref)
    lim = tol * bound + 1e-6
    bad = err > lim
    assert not bad.any(), (f"{bad.sum()} elements out of tolerance; worst "
                           f"{(err - lim).max():.3e} at {np.unravel_index(np.argmax(err - lim), err.shape)}")


@pytest.mark.parametrize("name", list(cases.CASES))
@pytest.mark.parametrize("N", [16, 64, 128])
def test_window_spmm_vs_fp64(cuda, name, N):
    from dtc_b200 import metcf
    rp, col, val, M, m, B, Bt = _setup(name, N)
    _check(metcf.spmm(m, Bt), rp, col, val, M, B)
    _check(metcf.spmm(m, Bt, use_values=False), rp, col, None, M, B)


@pytest.mark.parametrize("N", [4, 8, 20, 32, 36, 100, 132, 256, 260, 512, 600])
def test_window_spmm_widths(cuda, N):
    from dtc_b200 import metcf
    rp, col, val, M, m, B, Bt = _setup("wide_window", N)
    _check(metcf.spmm(m, Bt), rp, col, val, M, B)


@pytest.mark.parametrize("name", list(cases.CASES))
@pytest.mark.parametrize("N", [32, 128, 256])
def test_balance_spmm_vs_fp64_and_deterministic(cuda, name, N):
    from dtc_b200 import metcf
    rp, col, val, M, m, B, Bt = _setup(name, N)
    C1 = metcf.spmm_balance(m, Bt)
    C2 = metcf.spmm_balance(m, Bt)
    _check(C1, rp, col, val, M, B)
    assert (C1.view(-1).view(dtype=__import__("torch").int32) ==
            C2.view(-1).view(dtype=__import__("torch").int32)).all(), "balance SpMM not bitwise reproducible"


@pytest.mark.parametrize("grid", [1, 2, 3, 7, 33, 148, 1000])
@pytest.mark.parametrize("N", [64, 256, 600])
def test_schedules_across_many_boundaries(cuda, grid, N):
    # grid = 1 drives one CTA around its stage ring many times (every
    # barrier phase is reused); larger grids cut windows across CTAs
    from dtc_b200 import metcf, B_F32, PREC_TF32
    for name in ("hub", "banded_dense"):
        rp, col, val, M, m, B, Bt = _setup(name, N)
        C = metcf.spmm_ex(m, [Bt], B_F32, N, PREC_TF32, mode=1, grid=grid)
        _check(C, rp, col, val, M, B)
        Cw = metcf.spmm_ex(m, [Bt], B_F32, N, PREC_TF32, mode=0, grid=grid)
        _check(Cw, rp, col, val, M, B)
    assert metcf.device_status(clear=True) == 0


def test_empty_windows_are_zeroed(cuda):
    import torch
    from dtc_b200 import metcf
    rp, col, val, M, m, B, Bt = _setup("empty_windows", 32)
    for fn in (metcf.spmm, metcf.spmm_balance):
        out = torch.full((M, 32), float("nan"), device="cuda")
        C = fn(m, Bt, out=out)
        assert torch.isfinite(C).all()
        assert (C[16:48] == 0).all()
        _check(C, rp, col, val, M, B)


def test_all_ones_known_answer(cuda):
    import torch
    from dtc_b200 import metcf
    rp, col, val, M = cases.duplicates()
    m = metcf.convert(rp, col, M)
    X = torch.ones((M, 16), device="cuda")
    deg = np.array([len(set(col[rp[i]:rp[i + 1]])) for i in range(M)], np.float32)
    for C in (metcf.spmm(m, X), metcf.spmm_balance(m, X), metcf.spmm_mma_sync(m, X)):
        np.testing.assert_array_equal(C.cpu().numpy(), np.repeat(deg[:, None], 16, axis=1))


@pytest.mark.parametrize("N", [1, 5, 16, 33, 128, 300])
def test_mma_sync_kernel(cuda, N):
    from dtc_b200 import metcf
    rp, col, val, M, m, B, Bt = _setup("small_uniform", N)
    _check(metcf.spmm_mma_sync(m, Bt), rp, col, val, M, B)


@pytest.mark.parametrize("name", [n for n in cases.CASES])
def test_against_reference_spmm_golden(cuda, name):
    import torch
    from dtc_b200 import metcf
    path = os.path.join(GOLDEN, f"ref_gpu_{name}.npz")
    if not os.path.exists(path):
        pytest.skip("no reference golden vector")
    g = np.load(path)
    if "C_run" not in g.files and "C_run128" not in g.files:
        pytest.skip("reference SpMM not run on this case (num_nodes % 16 != 0)")
    rp, col, _, M = cases.CASES[name]()
    m = metcf.convert(rp, col, M)
    if "C_run" not in g.files:
        _check_reference_n128(m, rp, col, M, g)
        return
    Bt = torch.from_numpy(g["B"]).cuda()
    bound = O.spmm_absbound_f64(rp, col, None, M, g["B"])
    # The reference's balance launcher runs its atomicAdd-flushing kernel
    # EXE_TIME = 1000 times into one zero-filled output
    # (DTC-SpMM/DTCSpMM_kernel.cu:1118-1160, flush at :4885-4900), so the C it
    # returns is 1000 * A*B (summed in fp32); the window launcher overwrites.
    ref_balance = g["C_balance"].astype(np.float64) / 1000.0
    for ours in (metcf.spmm(m, Bt), metcf.spmm_balance(m, Bt)):
        o = ours.cpu().numpy().astype(np.float64)
        # both sides are TF32 products of the same operands
        assert (np.abs(o - g["C_run"]) <= 2 * TF32_TOL * bound + 1e-6).all(), "C_run"
        assert (np.abs(o - ref_balance) <= (2 * TF32_TOL + 1e-4) * bound + 1e-5).all(), \
            "C_balance"
    if "C_run128" not in g.files:
        return
    _check_reference_n128(m, rp, col, M, g)


def _check_reference_n128(m, rp, col, M, g):
    """N = 128 through the reference's float4_split plans, against both of ours
    and the FP64 product, on the rows the golden file keeps."""
    import torch
    from dtc_b200 import metcf
    from tests.golden import make_golden
    B = make_golden.b128(M)
    assert B.astype(np.float64).sum() == float(g["B128_sum"]), "B128 generator changed"
    rows = g["rows128"]
    Bt = torch.from_numpy(B).cuda()
    bound = O.spmm_absbound_f64(rp, col, None, M, B)[rows]
    c64 = O.spmm_f64(rp, col, None, M, B)[rows]
    ref_balance = g["C_balance128"].astype(np.float64) / 1000.0
    assert (np.abs(g["C_run128"] - c64) <= TF32_TOL * bound + 1e-6).all(), "reference C_run128"
    for ours in (metcf.spmm(m, Bt), metcf.spmm_balance(m, Bt)):
        o = ours.cpu().numpy().astype(np.float64)[rows]
        assert (np.abs(o - c64) <= TF32_TOL * bound + 1e-6).all(), "ours vs FP64"
        assert (np.abs(o - g["C_run128"]) <= 2 * TF32_TOL * bound + 1e-6).all(), "C_run128"
        assert (np.abs(o - ref_balance) <= (2 * TF32_TOL + 1e-4) * bound + 1e-5).all(), \
            "C_balance128"


def test_extension_api_matches_c_abi(cuda):
    import torch
    import DTCSpMM
    from dtc_b200 import metcf
    rp, col, val, M, m, B, Bt = _setup("hub", 128)
    ref_w = metcf.spmm(m, Bt, use_values=False)
    ref_b = metcf.spmm_balance(m, Bt, use_values=False)
    for plan in ("float_nonsplit", "float4_split", "float2_split"):
        C = DTCSpMM.run_DTCSpMM(Bt, m.RowWindowOffset, m.TCblocktileId, m.TCblockoffset,
                                m.SparseAToX, M, len(col), plan)[0]
        assert torch.equal(C, ref_w)
    C = DTCSpMM.DTCSpMM_gcn(Bt, m.RowWindowOffset, m.TCblocktileId, m.TCblockoffset,
                            m.SparseAToX, M, len(col))[0]
    assert torch.equal(C, ref_w)
    for plan in ("float_nonsplit", "float4_split"):
        C = DTCSpMM.run_DTCSpMM_balance(Bt, m.TCblockRowid, m.TCblocktileId, m.TCblockoffset,
                                        m.SparseAToX, M, plan)[0]
        assert torch.equal(C, ref_b)
    Cv = DTCSpMM.run_DTCSpMM(Bt, m.RowWindowOffset, m.TCblocktileId, m.TCblockoffset,
                             m.SparseAToX, M, len(col), "float_nonsplit", values=m.TCvalues)[0]
    assert torch.equal(Cv, metcf.spmm(m, Bt))
    with pytest.raises(RuntimeError):
        DTCSpMM.run_DTCSpMM(Bt, m.RowWindowOffset, m.TCblocktileId, m.TCblockoffset,
                            m.SparseAToX, M, len(col), "float8_magic")


def test_no_device_errors_recorded(cuda):
    from dtc_b200 import metcf
    assert metcf.device_status(clear=True) == 0


@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("form", ["tf32", "split24x4"])
@pytest.mark.parametrize("name", ["hub", "empty_windows", "small_uniform"])
def test_fused_bias_relu_epilogue(cuda, name, form, mode):
    """C = ReLU(A B + bias) from one launch, windows split across CTAs included."""
    import torch
    from dtc_b200 import metcf, tune
    rp, col, val, M = cases.CASES[name]()
    m = metcf.convert(rp, col, M, values=val)
    N = 64
    B = np.random.default_rng(11).standard_normal((M, N)).astype(np.float32)
    bias = np.random.default_rng(12).standard_normal(N).astype(np.float32)
    fmt, prec = tune.FORMS[form][0], tune.FORMS[form][1]
    Bd = torch.from_numpy(B).cuda()
    planes = [Bd] if form == "tf32" else metcf.pack_b(Bd, fmt)
    C = metcf.spmm_fused(m, planes, fmt, N, prec, bias=torch.from_numpy(bias).cuda(), relu=True,
                         mode=mode, grid=7 if mode else 0).cpu().numpy().astype(np.float64)
    ref = np.maximum(O.spmm_f64(rp, col, val, M, B) + bias, 0.0)
    bound = O.spmm_absbound_f64(rp, col, val, M, B)
    tol = 2.0 ** -9 if form == "tf32" else 2.0 ** -14
    assert (np.abs(C - ref) <= tol * bound + 1e-6).all()
    assert metcf.device_status(clear=True) == 0


def test_gcn_entry_bias_relu(cuda):
    import torch
    import DTCSpMM
    from dtc_b200 import metcf
    rp, col, _, M = cases.small_uniform()
    m = metcf.convert(rp, col, M)
    X = torch.randn(M, 32, device="cuda")
    b = torch.randn(32, device="cuda")
    (C,) = DTCSpMM.DTCSpMM_gcn(X, m.RowWindowOffset, m.TCblocktileId, m.TCblockoffset,
                               m.SparseAToX, M, len(col), bias=b, relu=True)
    (P,) = DTCSpMM.DTCSpMM_gcn(X, m.RowWindowOffset, m.TCblocktileId, m.TCblockoffset,
                               m.SparseAToX, M, len(col))
    torch.testing.assert_close(C, torch.relu(P + b), rtol=0, atol=1e-6)


def test_rowid_to_window_offset_matches_conversion(cuda):
    import ctypes as C
    import torch
    from dtc_b200 import _lib, metcf
    rp, col, val, M = cases.empty_windows()
    m = metcf.convert(rp, col, M, values=val)
    rwo = torch.full((m.nwin + 1,), -7, dtype=torch.int32, device="cuda")
    rc = _lib.lib().dtc_rowid_to_window_offset(
        C.c_void_p(m.TCblockRowid.data_ptr()), C.c_int64(m.T), m.nwin, C.c_void_p(rwo.data_ptr()),
        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    assert torch.equal(rwo, m.RowWindowOffset)
    assert metcf.device_status(clear=True) == 0


@pytest.mark.parametrize("bad", ["too_large", "negative", "descending"])
def test_rowid_to_window_offset_flags_bad_ids_and_stays_in_bounds(cuda, bad):
    """Window ids are caller input: ids outside [0, num_windows) or out of order
    set the device error bit for a skipped index, and the writes stay inside the
    (num_windows + 1)-entry table (canaries on both sides stay intact)."""
    import ctypes as C
    import torch
    from dtc_b200 import _lib, metcf
    nwin, T = 10, 40
    rowid = torch.arange(T, dtype=torch.int32, device="cuda") // 4
    if bad == "too_large":
        rowid[-3:] = nwin + 1000
    elif bad == "negative":
        rowid[:2] = -50
    else:
        rowid[20] = 1
    buf = torch.full((nwin + 1 + 64,), 12345, dtype=torch.int32, device="cuda")
    rwo = buf[32:32 + nwin + 1]
    metcf.device_status(clear=True)
    rc = _lib.lib().dtc_rowid_to_window_offset(
        C.c_void_p(rowid.data_ptr()), C.c_int64(T), nwin, C.c_void_p(rwo.data_ptr()),
        C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    assert metcf.device_status(clear=True) & 2
    assert (buf[:32] == 12345).all() and (buf[32 + nwin + 1:] == 12345).all()


def _long_hole(M=12000, seed=3):
    """Rows 1000..8999 empty (a run of 500 empty 16-row windows, longer than the
    kernels' window-record ring) plus scattered empty rows."""
    rng = np.random.default_rng(seed)
    rows = []
    for i in range(M):
        if 1000 <= i < 9000 or i % 17 == 5:
            rows.append(np.zeros(0, np.int64))
        else:
            rows.append(np.sort(rng.choice(M, size=int(rng.integers(1, 30)), replace=False)))
    rp = np.zeros(M + 1, np.int32)
    rp[1:] = np.cumsum([len(r) for r in rows])
    col = np.concatenate(rows).astype(np.int32)
    val = rng.uniform(-1, 1, len(col)).astype(np.float32)
    return rp, col, val, M


@pytest.mark.parametrize("H", [16, 32])
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("grid", [0, 5, 148])
def test_long_run_of_empty_windows(cuda, H, mode, grid):
    import torch
    from dtc_b200 import metcf, B_F32, B_BF16X2, PREC_TF32, PREC_SPLIT3
    rp, col, val, M = _long_hole()
    m = metcf.convert(rp, col, M, H=H, values=val)
    N = 64
    B = np.random.default_rng(4).standard_normal((M, N)).astype(np.float32)
    Bt = torch.from_numpy(B).cuda()
    ref = O.spmm_f64(rp, col, val, M, B)
    bound = O.spmm_absbound_f64(rp, col, val, M, B)
    for fmt, prec, tol in ((B_F32, PREC_TF32, TF32_TOL), (B_BF16X2, PREC_SPLIT3, 2.0 ** -14)):
        planes = [Bt] if fmt == B_F32 else metcf.pack_b(Bt, fmt)
        C = metcf.spmm_ex(m, planes, fmt, N, prec, mode=mode, grid=grid).cpu().numpy()
        assert (np.abs(C.astype(np.float64) - ref) <= tol * bound + 1e-6).all()
    assert metcf.device_status(clear=True) == 0


@pytest.mark.parametrize("mode", [0, 1])
def test_chunk_queue_and_one_cta_per_chunk_agree_bitwise(cuda, mode):
    """Persistent CTAs pulling chunks from the queue and one CTA per chunk give
    the same bits: results depend only on the chunking."""
    import torch
    from dtc_b200 import gen, metcf, B_F32, B_BF16X2, PREC_TF32, PREC_SPLIT3
    A = gen.rmat(14, 16.0, 0.57, 0.19, 0.19, seed=2)
    for H in (16, 32):
        m = metcf.convert(A.rowptr, A.col, A.M, H=H, values=A.val)
        N = 128
        Bt = torch.from_numpy(gen.normal(A.M, N, seed=1)).cuda()
        for fmt, prec in ((B_F32, PREC_TF32), (B_BF16X2, PREC_SPLIT3)):
            planes = [Bt] if fmt == B_F32 else metcf.pack_b(Bt, fmt)
            full = metcf.spmm_ex_workspace_bytes(m, N, mode, 0)
            queue = metcf.spmm_ex_workspace_bytes(m, N, 0, 0)  # the queue region alone
            outs = []
            for wsb in (full, full - queue):
                ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device="cuda")
                outs.append(metcf.spmm_ex(m, planes, fmt, N, prec, mode=mode, workspace=ws))
            assert torch.equal(outs[0], outs[1])
    assert metcf.device_status(clear=True) == 0
