"""The reference's own SpMM kernels, rebuilt for sm_100a (oracle/_ref/), beside
this library's on the same ME-TCF arrays (A = 1): both agree with the FP64
product within TF32 tolerance, and with each other. With DTC_REF_TIMING set to
a file path, the full-size R-MAT 2^20, N = 128 case also runs and its kernel
times are written there as JSON (the reference-on-B200 comparison)."""
import glob
import json
import os
import subprocess
import sys

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
HAVE_REF = bool(glob.glob(os.path.join(ROOT, "oracle", "_ref", "DTCSpMM*.so")))


def _run(tmp_path, scale, N, reps=20):
    out = tmp_path / f"ref_s{scale}_n{N}.npz"
    r = subprocess.run([sys.executable, os.path.join(HERE, "ref_kernels_runner.py"),
                        "--scale", str(scale), "--N", str(N), "--reps", str(reps),
                        "--out", str(out)], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return dict(np.load(out))


@pytest.mark.skipif(not HAVE_REF, reason="reference extension not built (oracle/_ref)")
def test_reference_kernels_agree(cuda, tmp_path):
    from dtc_b200 import gen
    res = _run(tmp_path, 13, 128)
    A = gen.rmat(13, 16.0, 0.57, 0.19, 0.19, seed=0)
    B = gen.normal(A.M, 128, seed=1)
    ones = np.ones(A.nnz, np.float32)
    ref = O.spmm_f64(A.rowptr, A.col, ones, A.M, B)
    bound = O.spmm_absbound_f64(A.rowptr, A.col, ones, A.M, B)
    assert int(res["device_status"]) == 0
    # the reference's balance entry zero-fills C once per call and then runs its
    # 1000 timing launches, each adding its partial rows with atomicAdd
    # (DTCSpMM_kernel.cu:1130, :1141-1180): its C holds 1000 x the product
    res["ref_balance_float4_split_C"] = res["ref_balance_float4_split_C"] / 1000.0
    for k in ("ref_window_float_nonsplit_C", "ref_window_float4_split_C",
              "ref_balance_float4_split_C", "ours_window_C", "ours_balance_C"):
        err = np.abs(res[k].astype(np.float64) - ref)
        assert (err <= 2.0 ** -9 * bound + 1e-6).all(), k
    # the two implementations differ only by tf32 rounding of B (rna vs truncation)
    d = np.abs(res["ours_window_C"].astype(np.float64) - res["ref_window_float4_split_C"])
    assert (d <= 2.0 ** -8 * bound + 1e-6).all()


@pytest.mark.skipif(not HAVE_REF or not os.environ.get("DTC_REF_TIMING"),
                    reason="full-size reference timing runs only when DTC_REF_TIMING is set")
def test_reference_timing_full_size(cuda, tmp_path):
    res = _run(tmp_path, 20, 128, reps=20)
    flops = 2.0 * float(res["nnz"]) * 128
    times = {k[:-3]: float(v) for k, v in res.items() if k.endswith("_ms")}
    rec = {"workload": "rmat-2^20-sym, A = 1, N = 128", "nnz": int(res["nnz"]),
           "T": int(res["T"]), "ms": times,
           "gflops": {k: flops / (v * 1e-3) / 1e9 for k, v in times.items()}}
    with open(os.environ["DTC_REF_TIMING"], "w") as f:
        json.dump(rec, f, indent=1)
    assert int(res["device_status"]) == 0
