"""CPU tests of the C-ABI boundary: the library loads, exports every symbol the
headers declare, and rejects bad arguments with a status (never exits)."""
import ctypes as C
import os
import re

import pytest

from dtc_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if not f.endswith(".h"):
            continue
        src = open(os.path.join(inc, f)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(dtc_[a-z0-9_]+)\s*\(", src))
    return names


def test_header_declares_entry_points():
    d = _declared()
    for n in ("dtc_convert_count", "dtc_convert_fill", "dtc_spmm", "dtc_spmm_balance"):
        assert n in d


def test_library_exports_every_declared_symbol():
    L = C.CDLL(_lib.LIBDTC_PATH)
    missing = [n for n in sorted(_declared()) if not hasattr(L, n)]
    assert not missing, missing


def test_python_binding_covers_every_declared_symbol():
    assert _declared() <= set(_lib.SIGNATURES)


def test_version_and_error_text():
    assert _lib.lib().dtc_version() >= 100
    assert isinstance(_lib.lib().dtc_last_error(), bytes)


def test_bad_arguments_return_status_not_exit():
    L = _lib.lib()
    n = C.c_size_t()
    assert L.dtc_convert_workspace_bytes(-1, 10, 16, 8, C.byref(n)) == 1
    assert b"negative" in L.dtc_last_error()
    assert L.dtc_convert_workspace_bytes(10, 10, 32, 16, C.byref(n)) == 1  # 32*16 > 256
    assert L.dtc_bformat_bytes(99, 10, 10, C.byref(n), C.byref(n)) == 1
    assert L.dtc_spmm(None, None, None, None, None, 16, 1, 1, None, 16, None, None) == 1
    assert L.dtc_spmm_ex(None, None, None, None, None, 16, 1, 1, 16, 8, 0, None, None, 16, 0,
                         None, 7, 0, 0, None, 0, None) == 1
    assert L.dtc_tca_merge(None, None, 3, None, 0, 4, None) == 1  # host entry: null sets
    assert b"null" in L.dtc_last_error()
    assert L.dtc_tca_merge(None, None, 0, None, 0, 4, None) == 0  # no items: nothing to do


def test_bformat_sizes():
    L = _lib.lib()
    a, b = C.c_size_t(), C.c_size_t()
    assert L.dtc_bformat_bytes(_lib.B_SPLIT24, 10, 128, C.byref(a), C.byref(b)) == 0
    assert (a.value, b.value) == (2560, 1280)  # 3 bytes / element
    assert L.dtc_bformat_bytes(_lib.B_FP8, 10, 128, C.byref(a), C.byref(b)) == 0
    assert (a.value, b.value) == (1280, 40)


def test_torch_extension_mirrors_reference_api():
    pytest.importorskip("torch")
    import DTCSpMM
    for n in ("preprocess_gpu", "run_DTCSpMM", "run_DTCSpMM_balance", "DTCSpMM_gcn",
              "backward_ptx_uint8_improved", "backward_ptx_uint8_improved_gcn",
              "balance_backward_ptx_uint8_prefetch"):
        assert hasattr(DTCSpMM, n), n
    assert os.path.dirname(DTCSpMM.__file__) == os.path.dirname(os.path.dirname(_lib.LIBDTC_PATH))
