"""Generates the golden vectors of tests/golden/ from the reference itself.

The reference extension is built unmodified from its sources by
``oracle/build_ref.py`` into ``oracle/_ref/`` (test infrastructure only).

  --cpu  (any machine with the built reference): runs the reference's CPU
         ``preprocess`` (DTC-SpMM/DTCSpMM.cpp:233-311) on the cases it handles
         safely and stores blockPartition / edgeToColumn / edgeToRow in
         ref_cpu_<case>.npz.
  --gpu  (needs a CUDA device): runs the reference's ``preprocess_gpu``
         (DTCSpMM.cpp:313-359) on every case at every block shape of
         cases.GOLDEN_SHAPES (blockSize_h x blockSize_w = 16 x 8, 32 x 8,
         16 x 16; the reference takes both as arguments, DTCSpMM.cpp:315-316)
         and stores all ME-TCF arrays in the file cases.golden_name() names;
         at 16 x 8, for cases with num_nodes % 16 == 0 (the reference SpMM
         kernels store 16 rows per window without a bound check,
         DTCSpMM_kernel.cu:2850-2865) it also stores the reference SpMM output
         of run_DTCSpMM / run_DTCSpMM_balance with 'float_nonsplit' for
         B = seeded N(0,1) with N = 32 and with 'float4_split' for N = 128
         (A = 1); see compact() for what is kept of the N = 128 products.

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
import cases  # noqa: E402


def _reference_module():
    """The reference extension built into oracle/_ref, loaded from its file
    (never through sys.path: importing this module must not shadow the
    library's own DTCSpMM module of the same name). A process holds one
    extension module per name, so call this only in a process that does not
    use the library's DTCSpMM module (this script run on its own)."""
    import glob
    import importlib.util
    found = glob.glob(os.path.join(ROOT, "oracle", "_ref", "DTCSpMM*.so"))
    if not found:
        raise RuntimeError("reference extension not built (python oracle/build_ref.py)")
    spec = importlib.util.spec_from_file_location("DTCSpMM", found[0])
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


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
    DTCSpMM = _reference_module()
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


def b128(M):
    """The N = 128 operand of the reference SpMM goldens (regenerated, not stored)."""
    return np.random.default_rng(4321).standard_normal((M, 128)).astype(np.float32)


def sampled_rows(M):
    """Rows of every 8th 16-row window: where the N = 128 outputs are stored."""
    return np.concatenate([np.arange(w, min(w + 16, M)) for w in range(0, M, 128)])


def compact(name, arrays):
    """Keeps the files small: B128 is replaced by its checksum, the N = 128
    outputs are kept on sampled_rows(), and the power-law case carries only its
    N = 128 products."""
    if "B128" in arrays:
        B = arrays.pop("B128")
        rows = sampled_rows(B.shape[0])
        arrays["B128_sum"] = np.float64(B.astype(np.float64).sum())
        arrays["rows128"] = rows
        for k in ("C_run128", "C_balance128"):
            arrays[k] = arrays[k][rows]
    if name == "rmat12":
        for k in ("B", "C_run", "C_balance"):
            arrays.pop(k, None)
    return arrays


def gen_gpu(out, shapes, names):
    import torch
    DTCSpMM = _reference_module()
    dev = torch.device("cuda")
    for name in names:
        rp, col, _, M = cases.CASES[name]()
        for H, W in shapes:
            nwin = (M + H - 1) // H
            bp = torch.zeros(nwin, dtype=torch.int32, device=dev)
            e2c = torch.zeros(len(col), dtype=torch.int32, device=dev)
            e2r = torch.zeros(len(col), dtype=torch.int32, device=dev)
            rwo, rowid, tile, toff, s2x, T = DTCSpMM.preprocess_gpu(
                torch.from_numpy(col).to(dev), torch.from_numpy(rp).to(dev), M, H, W, bp, e2c,
                e2r)
            arrays = dict(T=np.int64(T), RowWindowOffset=rwo.cpu().numpy(),
                          TCblockRowid=rowid.cpu().numpy(), TCblocktileId=tile.cpu().numpy(),
                          TCblockoffset=toff.cpu().numpy(), SparseAToX=s2x.cpu().numpy(),
                          blockPartition=bp.cpu().numpy(), edgeToColumn=e2c.cpu().numpy(),
                          edgeToRow=e2r.cpu().numpy())
            # the reference SpMM kernels are written for 16 x 8 blocks
            if (H, W) == (16, 8) and M % 16 == 0 and T > 0:
                rng = np.random.default_rng(1234)
                B = rng.standard_normal((M, 32)).astype(np.float32)
                X = torch.from_numpy(B).to(dev)
                with _in_tmpdir():
                    C1 = DTCSpMM.run_DTCSpMM(X, rwo, tile, toff, s2x, M, len(col),
                                             "float_nonsplit")[0]
                    C2 = DTCSpMM.run_DTCSpMM_balance(X, rowid, tile, toff, s2x, M,
                                                     "float_nonsplit")[0]
                torch.cuda.synchronize()
                arrays.update(B=B, C_run=C1.cpu().numpy(), C_balance=C2.cpu().numpy())
                # N = 128 through the plans the reference's schedule table uses
                # for N = 128 (scripts/DTCSpMM/run_DTC_SpMM.py:10-21)
                B128 = b128(M)
                X = torch.from_numpy(B128).to(dev)
                with _in_tmpdir():
                    C3 = DTCSpMM.run_DTCSpMM(X, rwo, tile, toff, s2x, M, len(col),
                                             "float4_split")[0]
                    C4 = DTCSpMM.run_DTCSpMM_balance(X, rowid, tile, toff, s2x, M,
                                                     "float4_split")[0]
                torch.cuda.synchronize()
                arrays.update(B128=B128, C_run128=C3.cpu().numpy(),
                              C_balance128=C4.cpu().numpy())
            np.savez_compressed(os.path.join(out, cases.golden_name(name, H, W)),
                                **compact(name, arrays))
            print("gpu", name, H, W, T)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--cpu", action="store_true")
    ap.add_argument("--gpu", action="store_true")
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--shapes", default=",".join(f"{h}x{w}" for h, w in cases.GOLDEN_SHAPES),
                    help="block shapes HxW for --gpu, comma-separated")
    ap.add_argument("--cases", default=",".join(cases.CASES), help="case names for --gpu")
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    if a.cpu:
        gen_cpu(a.out)
    if a.gpu:
        shapes = [tuple(int(x) for x in t.split("x")) for t in a.shapes.split(",")]
        gen_gpu(a.out, shapes, a.cases.split(","))
