"""GPU test of dtc_spmm_balance_noalloc, the strict-balance SpMM for callers that
cannot allocate device memory (servers whose device memory belongs to their
own budgeted pool, plugins without an allocator): it keeps its scratch in an array compiled into
the library instead of a caller workspace.

Called through the C ABI and compared, within the TF32 tolerance of
tests/test_spmm_gpu.py, with the regular entry point (dtc_spmm_balance) and
with the FP64 product of the host oracle, on two calls in a row (the second
call reuses the array the first one left behind).
This file is named so that pytest collects it last; it also passes alone in a
fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tests.golden import cases

pytestmark = pytest.mark.gpu

TF32_TOL = 2.0 ** -9


def _ptr(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def _noalloc(m, B, out, stream):
    from dtc_b200 import _lib
    return _lib.lib().dtc_spmm_balance_noalloc(
        _ptr(m.TCblockRowid), _ptr(m.TCblocktileId), _ptr(m.TCblockoffset),
        _ptr(m.SparseAToX), _ptr(m.TCvalues), m.M, m.T, _ptr(B), B.shape[1], _ptr(out), stream)


@pytest.mark.parametrize("name,N", [("hub", 128), ("banded_dense", 256), ("empty_windows", 32),
                                    ("wide_window", 36)])
def test_noalloc_matches_workspace_entry_point_twice(cuda, name, N):
    import torch
    from dtc_b200 import _lib, metcf
    rp, col, val, M = cases.CASES[name]()
    m = metcf.convert(rp, col, M, values=val)
    B = np.random.default_rng(9).standard_normal((M, N)).astype(np.float32)
    Bt = torch.from_numpy(B).cuda()
    ref = metcf.spmm_balance(m, Bt).cpu().numpy().astype(np.float64)
    c64 = O.spmm_f64(rp, col, val, M, B)
    bound = O.spmm_absbound_f64(rp, col, val, M, B)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        out = torch.full((M, N), float("nan"), device="cuda")
        rc = _noalloc(m, Bt, out, stream)
        assert rc == 0, _lib.lib().dtc_last_error()
        got = out.cpu().numpy().astype(np.float64)
        assert np.isfinite(got).all()
        assert (np.abs(got - c64) <= TF32_TOL * bound + 1e-6).all(), f"call {call} vs FP64"
        assert (np.abs(got - ref) <= TF32_TOL * bound + 1e-6).all(), f"call {call}"
    assert metcf.device_status(clear=True) == 0


def test_noalloc_rejects_sizes_beyond_the_array(cuda):
    import torch
    from dtc_b200 import _lib, metcf
    rp, col, val, M = cases.hub()
    m = metcf.convert(rp, col, M, values=val)
    cap = _lib.lib().dtc_noalloc_scratch_capacity()
    N = 1024  # 128 * N bytes per SM of partial tiles exceeds 16 MiB on 148 SMs
    assert 128 * N * torch.cuda.get_device_properties(0).multi_processor_count > cap
    B = torch.zeros((M, N), device="cuda")
    out = torch.zeros((M, N), device="cuda")
    rc = _noalloc(m, B, out, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 2  # DTC_ERR_WORKSPACE_TOO_SMALL
    assert b"scratch" in _lib.lib().dtc_last_error()
