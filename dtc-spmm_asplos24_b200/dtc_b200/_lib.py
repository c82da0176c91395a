"""ctypes binding of the C ABI (include/dtc_spmm.h, lib/libdtcspmm.so).

Every exported symbol is declared here with its argument types; ``call``
raises ``DtcError`` with the library's error text on a non-zero status. No
computation happens in Python: when the library is missing the import fails
loudly (there is no fallback path).
"""
import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_DIR = os.path.join(PKG_DIR, "lib")
LIBDTC_PATH = os.path.join(LIB_DIR, "libdtcspmm.so")
LIBGEN_PATH = os.path.join(LIB_DIR, "libdtcgen.so")

i32, i64, u64, f64 = C.c_int32, C.c_int64, C.c_uint64, C.c_double
vp, sz = C.c_void_p, C.c_size_t
szp = C.POINTER(C.c_size_t)
i64p = C.POINTER(C.c_int64)
u32p = C.POINTER(C.c_uint32)

# name -> argtypes (restype is dtc_status == int unless listed in _RESTYPES)
SIGNATURES = {
    "dtc_last_error": [],
    "dtc_version": [],
    "dtc_device_status": [u32p, C.c_int],
    "dtc_convert_workspace_bytes": [i32, i64, i32, i32, szp],
    "dtc_convert_count": [vp, vp, i32, i64, i32, i32, vp, vp, vp, vp, vp, sz, i64p, vp],
    "dtc_convert_fill": [vp, vp, i32, i64, i32, i32, vp, vp, vp, i64, vp, vp, vp, vp, vp, vp,
                         vp, sz, vp],
    "dtc_bformat_bytes": [C.c_int, i64, i32, szp, szp],
    "dtc_pack_b": [C.c_int, vp, i64, i32, vp, vp, vp],
    "dtc_spmm": [vp, vp, vp, vp, vp, i32, i32, i64, vp, i32, vp, vp],
    "dtc_spmm_balance_workspace_bytes": [i32, i64, i32, szp],
    "dtc_spmm_balance": [vp, vp, vp, vp, vp, i32, i64, vp, i32, vp, vp, sz, vp],
    "dtc_spmm_ex": [vp, vp, vp, vp, vp, i32, i32, i64, i32, i32, C.c_int, vp, vp, i32, C.c_int,
                    vp, C.c_int, C.c_int, C.c_int, vp, sz, vp],
    "dtc_spmm_ex_workspace_bytes": [i32, i64, i32, i32, C.c_int, C.c_int, szp],
    "dtc_spmm_fused": [vp, vp, vp, vp, vp, i32, i32, i64, i32, i32, C.c_int, vp, vp, i32,
                       C.c_int, vp, C.c_int, vp, C.c_int, C.c_int, C.c_int, vp, sz, vp],
    "dtc_rowid_to_window_offset": [vp, i64, i32, vp, vp],
    "dtc_set_cta_timer": [vp, i32],
    "dtc_spmm_mma_sync": [vp, vp, vp, vp, vp, i32, i32, vp, i32, vp, vp],
    "dtc_spmm_balance_noalloc": [vp, vp, vp, vp, vp, i32, i64, vp, i32, vp, vp],
    "dtc_noalloc_scratch_capacity": [],
    "dtc_schedule_candidates": [i32, vp, C.c_int],
    "dtc_schedule_candidates_ex": [i32, i32, C.c_int, vp, C.c_int],
    "dtc_relabel_workspace_bytes": [i32, i32, i64, szp],
    "dtc_tca_default_params": [vp],
    "dtc_features_workspace_bytes": [],
    "dtc_features": [vp, vp, i32, i64, vp, vp, vp, i32, i64, i32, vp, vp, sz, vp],
    "dtc_mlp_num_params": [vp],
    "dtc_mlp_forward": [vp, vp, vp, i32, vp, vp, vp, vp],
    "dtc_mlp_backward_workspace_bytes": [vp, i32],
    "dtc_mlp_backward": [vp, vp, vp, vp, vp, vp, vp, vp, i32, vp, vp, vp, sz, vp],
    "dtc_mlp_adam": [vp, vp, vp, vp, i64, C.c_float, C.c_float, C.c_float, C.c_float, i32, vp],
    "dtc_mlp_argmin": [vp, vp, C.c_int, i32, i32, vp, vp],
    "dtc_tca_workspace_bytes": [i32, i64, vp, szp],
    "dtc_tca_reorder": [vp, vp, i32, i64, vp, vp, vp, sz, vp],
    "dtc_tca_merge": [vp, vp, i32, vp, i64, i32, vp],
    "dtc_permute_csr": [vp, vp, vp, i32, i64, vp, vp, vp, vp, i64p, vp, sz, vp],
    "dtc_transpose_csr": [vp, vp, vp, i32, i32, i64, vp, vp, vp, i64p, vp, sz, vp],
    "dtc_coo_to_csr": [vp, vp, vp, i32, i32, i64, vp, vp, vp, i64p, vp, sz, vp],
    "dtc_autotune_workspace_bytes": [i32, i64, i32, i32, szp],
    "dtc_autotune": [vp, vp, vp, vp, vp, i32, i32, i64, i32, i32, C.c_int, vp, vp, i32, C.c_int,
                     vp, vp, sz, C.c_int, vp, C.c_int, vp, vp, vp],
}
_RESTYPES = {"dtc_last_error": C.c_char_p, "dtc_version": C.c_int,
             "dtc_noalloc_scratch_capacity": C.c_size_t, "dtc_schedule_candidates": C.c_int,
             "dtc_schedule_candidates_ex": C.c_int,
             "dtc_tca_default_params": None, "dtc_features_workspace_bytes": C.c_size_t,
             "dtc_mlp_num_params": C.c_int64, "dtc_mlp_backward_workspace_bytes": C.c_size_t}


class MlpDims(C.Structure):
    """dtc_mlp_dims (include/dtc_spmm.h)."""
    _fields_ = [("in_", C.c_int32), ("h1", C.c_int32), ("h2", C.c_int32), ("out", C.c_int32)]


class TcaParams(C.Structure):
    """dtc_tca_params (include/dtc_spmm.h)."""
    _fields_ = [("num_perm", C.c_int32), ("bands", C.c_int32), ("rows_per_band", C.c_int32),
                ("thres", C.c_int32), ("c_thres", C.c_int32), ("bucket_window", C.c_int32),
                ("seed", C.c_uint64)]


class Schedule(C.Structure):
    """dtc_schedule (include/dtc_spmm.h)."""
    _fields_ = [("mode", C.c_int32), ("waves", C.c_int32), ("ntile", C.c_int32),
                ("grid", C.c_int32), ("ms", C.c_float)]

    def key(self):
        return (self.mode, self.waves, self.ntile)

    def __repr__(self):
        return (f"Schedule(mode={self.mode}, waves={self.waves}, ntile={self.ntile}, "
                f"grid={self.grid}, ms={self.ms:.4f})")

B_F32, B_SPLIT24, B_BF16, B_FP8, B_BF16X2 = 0, 1, 2, 3, 4
PREC_TF32, PREC_SPLIT3, PREC_SPLIT4 = 0, 1, 2


class DtcError(RuntimeError):
    pass


_lib = None
_gen = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIBDTC_PATH):
            raise ImportError(f"{LIBDTC_PATH} is not built; run dtc-spmm_asplos24_b200/build.py")
        L = C.CDLL(LIBDTC_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, C.c_int)
        _lib = L
    return _lib


def call(name, *args):
    rc = getattr(lib(), name)(*args)
    if rc != 0:
        msg = lib().dtc_last_error().decode(errors="replace")
        raise DtcError(f"{name} -> status {rc}: {msg}")
    return rc


def gen():
    global _gen
    if _gen is None:
        if not os.path.exists(LIBGEN_PATH):
            raise ImportError(f"{LIBGEN_PATH} is not built; run dtc-spmm_asplos24_b200/build.py")
        G = C.CDLL(LIBGEN_PATH)
        G.dtcgen_uniform.argtypes = [i32, i32, f64, u64]
        G.dtcgen_rmat.argtypes = [i32, f64, f64, f64, f64, u64]
        G.dtcgen_stencil27.argtypes = [i32, u64]
        G.dtcgen_zipf.argtypes = [i32, f64, i32, i32, u64]
        G.dtcgen_banded.argtypes = [i32, i32, f64, u64]
        G.dtcgen_blockdiag.argtypes = [i32, i32, i32, f64, u64]
        for n in ("uniform", "rmat", "stencil27", "zipf", "banded", "blockdiag"):
            getattr(G, "dtcgen_" + n).restype = vp
        G.dtcgen_shape.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i64)]
        G.dtcgen_shape.restype = None
        G.dtcgen_copy.argtypes = [vp, vp, vp, vp]
        G.dtcgen_copy.restype = None
        G.dtcgen_free.argtypes = [vp]
        G.dtcgen_free.restype = None
        G.dtcgen_normal.argtypes = [vp, i64, u64]
        G.dtcgen_normal.restype = None
        _gen = G
    return _gen
