"""Generates the golden vectors of tests/golden/ from the reference itself.

The reference extension is built unmodified from its sources by
``oracle/build_ref.py`` into ``oracle/_ref/`` (test infrastructure only).

  --cpu  (any machine with the built reference): runs the reference's CPU
         ``preprocess`` (DTC-SpMM/DTCSpMM.cpp:233-311) on the cases it handles
         safely and stores blockPartition / edgeToColumn / edgeToRow in
         ref_cpu_<case>.npz.
  --gpu  (needs a CUDA device): runs the reference's ``preprocess_gpu``
         (DTCSpMM.cpp:313-359) on every case and stores all ME-TCF arrays in
         ref_gpu_<case>.npz; for cases with num_nodes % 16 == 0 (the reference
         SpMM kernels store 16 rows per window without a bound check,
         DTCSpMM_kernel.cu:2850-2865) it also stores the reference SpMM output
         of run_DTCSpMM('float_nonsplit') and run_DTCSpMM_balance
         ('float_nonsplit') for B = seeded N(0,1) with N = 32 (A = 1).

Outputs are written to the directory given by --out (default: this folder).
"""
import argparse
import contextlib
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
import cases  # noqa: E402


@contextlib.contextmanager
def _in_tmpdir():
    # the reference appends CSV rows to its working directory
    old = os.getcwd()
    with tempfile.TemporaryDirectory() as d:
        os.chdir(d)
        try:
            yield
        finally:
            os.chdir(old)


def gen_cpu(out):
    import torch
    import DTCSpMM
    for name in cases.CPU_REFERENCE_SAFE:
        rp, col, _, M = cases.CASES[name]()
        nwin = (M + 15) // 16
        # one extra slot: the reference writes blockPartition[nwin] when M % 16 == 0
        bp = torch.zeros(nwin + 1, dtype=torch.int32)
        e2c = torch.zeros(len(col), dtype=torch.int32)
        e2r = torch.zeros(len(col), dtype=torch.int32)
        T = DTCSpMM.preprocess(torch.from_numpy(col), torch.from_numpy(rp), M, 16, 8, bp, e2c, e2r)
        np.savez_compressed(os.path.join(out, f"ref_cpu_{name}.npz"), T=np.int64(T),
                            blockPartition=bp[:nwin].numpy(), edgeToColumn=e2c.numpy(),
                            edgeToRow=e2r.numpy())
        print("cpu", name, T)


def gen_gpu(out):
    import torch
    import DTCSpMM
    for name, fn in cases.CASES.items():
        rp, col, _, M = fn()
        nwin = (M + 15) // 16
        dev = torch.device("cuda")
        bp = torch.zeros(nwin, dtype=torch.int32, device=dev)
        e2c = torch.zeros(len(col), dtype=torch.int32, device=dev)
        e2r = torch.zeros(len(col), dtype=torch.int32, device=dev)
        rwo, rowid, tile, toff, s2x, T = DTCSpMM.preprocess_gpu(
            torch.from_numpy(col).to(dev), torch.from_numpy(rp).to(dev), M, 16, 8, bp, e2c, e2r)
        arrays = dict(T=np.int64(T), RowWindowOffset=rwo.cpu().numpy(),
                      TCblockRowid=rowid.cpu().numpy(), TCblocktileId=tile.cpu().numpy(),
                      TCblockoffset=toff.cpu().numpy(), SparseAToX=s2x.cpu().numpy(),
                      blockPartition=bp.cpu().numpy(), edgeToColumn=e2c.cpu().numpy(),
                      edgeToRow=e2r.cpu().numpy())
        if M % 16 == 0 and T > 0:
            N = 32
            B = np.random.default_rng(1234).standard_normal((M, N)).astype(np.float32)
            X = torch.from_numpy(B).to(dev)
            with _in_tmpdir():
                C1 = DTCSpMM.run_DTCSpMM(X, rwo, tile, toff, s2x, M, len(col), "float_nonsplit")[0]
                C2 = DTCSpMM.run_DTCSpMM_balance(X, rowid, tile, toff, s2x, M,
                                                 "float_nonsplit")[0]
            torch.cuda.synchronize()
            arrays.update(B=B, C_run=C1.cpu().numpy(), C_balance=C2.cpu().numpy())
        np.savez_compressed(os.path.join(out, f"ref_gpu_{name}.npz"), **arrays)
        print("gpu", name, T)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--cpu", action="store_true")
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--out", default=HERE)
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.cpu:
        gen_cpu(a.out)
    if a.gpu:
        gen_gpu(a.out)
