"""Runs the reference's own SpMM kernels, rebuilt unmodified for sm_100a into
oracle/_ref/ (test infrastructure), beside this library's kernels on the same
ME-TCF arrays, in a process of its own (both extension modules are named
DTCSpMM, so they cannot share a process).

The inputs are the seeded R-MAT family (a, b, c, d) = (0.57, 0.19, 0.19,
0.05), symmetrised with self-loops, at 2^scale nodes (a multiple of 16: the
reference's window kernels store 16 rows per window without a row bound,
DTC-SpMM/DTCSpMM_kernel.cu:4057-4074), and B = N(0,1). A = 1 for both sides,
because the reference ignores values (DTCSpMM_kernel.cu:837-838).

The reference times itself over 1000 back-to-back launches per call
(DTCSpMM_kernel.cu:18, :840-930); this runner brackets one such call with CUDA
events and divides by 1000 (kernel-only, like the reference). This library's
kernels are timed over `--reps` launches with CUDA events.

usage: python tests/ref_kernels_runner.py --scale S --N N --out result.npz [--reps R]
"""
import argparse
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "dtc-spmm_asplos24_b200")
REF = os.path.join(ROOT, "oracle", "_ref")
REF_LAUNCHES = 1000


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=14)
    ap.add_argument("--N", type=int, default=128)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--out", required=True)
    a = ap.parse_args()
    sys.path.insert(0, PKG)
    sys.path.insert(0, REF)  # the reference module wins the name DTCSpMM here
    import torch
    import DTCSpMM as ref
    assert os.path.dirname(os.path.abspath(ref.__file__)) == REF, ref.__file__
    from dtc_b200 import gen, metcf

    A = gen.rmat(a.scale, 16.0, 0.57, 0.19, 0.19, seed=0)
    assert A.M % 16 == 0
    N = a.N
    m = metcf.convert(A.rowptr, A.col, A.M)  # A = 1 (no values)
    X = torch.from_numpy(gen.normal(A.M, N, seed=1)).cuda()
    out = {"M": A.M, "nnz": A.nnz, "N": N, "T": m.T}

    def ev_time(fn, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(n):
            r = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n, r

    old = os.getcwd()
    with tempfile.TemporaryDirectory() as d:
        os.chdir(d)  # the reference appends a CSV row to its working directory
        try:
            for plan in ("float_nonsplit", "float4_split"):
                ref.run_DTCSpMM(X, m.RowWindowOffset, m.TCblocktileId, m.TCblockoffset,
                                m.SparseAToX, A.M, A.nnz, plan)  # warm-up call
                ms, (C,) = ev_time(lambda: ref.run_DTCSpMM(
                    X, m.RowWindowOffset, m.TCblocktileId, m.TCblockoffset, m.SparseAToX,
                    A.M, A.nnz, plan), 1)
                out[f"ref_window_{plan}_ms"] = ms / REF_LAUNCHES
                out[f"ref_window_{plan}_C"] = C.cpu().numpy()
            plan = "float4_split"
            ref.run_DTCSpMM_balance(X, m.TCblockRowid, m.TCblocktileId, m.TCblockoffset,
                                    m.SparseAToX, A.M, plan)
            ms, (C,) = ev_time(lambda: ref.run_DTCSpMM_balance(
                X, m.TCblockRowid, m.TCblocktileId, m.TCblockoffset, m.SparseAToX, A.M, plan), 1)
            out["ref_balance_float4_split_ms"] = ms / REF_LAUNCHES
            out["ref_balance_float4_split_C"] = C.cpu().numpy()
        finally:
            os.chdir(old)

    Cw = torch.empty_like(X)
    ms, _ = ev_time(lambda: metcf.spmm(m, X, use_values=False, out=Cw), a.reps)
    out["ours_window_ms"] = ms
    out["ours_window_C"] = Cw.cpu().numpy()
    ws = torch.empty(max(metcf.spmm_balance_workspace_bytes(m, N), 1), dtype=torch.uint8,
                     device="cuda")
    Cb = torch.empty_like(X)
    ms, _ = ev_time(lambda: metcf.spmm_balance(m, X, use_values=False, out=Cb, workspace=ws),
                    a.reps)
    out["ours_balance_ms"] = ms
    out["ours_balance_C"] = Cb.cpu().numpy()
    out["device_status"] = metcf.device_status(clear=True)
    np.savez(a.out, **out)


if __name__ == "__main__":
    main()
