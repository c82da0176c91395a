"""Runs one SpMM configuration a few times: a fixed target for profilers.

    python -m dtc_b200.profile --scale 19 --form bf16x2x3 --H 32 --mode 0 --reps 3

Builds the seeded R-MAT(0.57, 0.19, 0.19, 0.05) matrix of 2^scale nodes
(symmetrised, self-loops, GCN values; --stencil 126 for the 27-point stencil
instead), converts it to ME-TCF of block shape H x W, packs a seeded N(0,1)
B into the form's storage, runs --warmup untimed products and --reps timed
ones, and prints one JSON line with the mean CUDA-event time per product.
With --kernel pack or --kernel convert it repeats the B pack or the ME-TCF
conversion instead. Nothing else runs on the GPU, so a profiler's kernel
filter (for example ``ncu -k regex:k_spmm -c 1``) lands on the product.
"""
import argparse
import json
import time

import numpy as np
import torch

from . import gen, metcf, tune
from ._lib import B_F32


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--scale", type=int, default=19)
    ap.add_argument("--stencil", type=int, default=0)
    ap.add_argument("--N", type=int, default=128)
    ap.add_argument("--form", default="bf16x2x3", choices=list(tune.FORMS))
    ap.add_argument("--H", type=int, default=32)
    ap.add_argument("--W", type=int, default=8)
    ap.add_argument("--mode", type=int, default=0)
    ap.add_argument("--waves", type=int, default=16)
    ap.add_argument("--ntile", type=int, default=0)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--kernel", default="spmm", choices=["spmm", "pack", "convert"])
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    if a.stencil:
        A = gen.stencil27(a.stencil, seed=0)
        name = f"stencil27-{a.stencil}^3"
    else:
        A = gen.rmat(a.scale, 16.0, 0.57, 0.19, 0.19, seed=0)
        name = f"rmat-2^{a.scale}-sym-gcn"
    rp = torch.from_numpy(A.rowptr).to(dev)
    col = torch.from_numpy(A.col).to(dev)
    val = torch.from_numpy(A.val).to(dev)
    m = metcf.convert(rp, col, A.M, H=a.H, W=a.W, values=val, device=dev)
    B = torch.from_numpy(gen.normal(A.K, a.N, seed=1)).to(dev)
    fmt, prec = tune.FORMS[a.form][0], tune.FORMS[a.form][1]
    planes = [B] if fmt == B_F32 else metcf.pack_b(B, fmt)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    grid = min(a.waves * sms, max(m.T, 1))
    out = torch.empty((A.M, a.N), dtype=torch.float32, device=dev)
    ws = torch.empty(max(metcf.spmm_ex_workspace_bytes(m, a.N, a.mode, grid), 1),
                     dtype=torch.uint8, device=dev)
    if a.kernel == "spmm":
        fn = lambda: metcf.spmm_ex(m, planes, fmt, a.N, prec, mode=a.mode, grid=grid, out=out,
                                   workspace=ws, ntile=a.ntile)
    elif a.kernel == "pack":
        fn = lambda: metcf.pack_b_into(B, fmt, planes)
    else:
        fn = lambda: metcf.convert(rp, col, A.M, H=a.H, W=a.W, values=val, device=dev)
    for _ in range(a.warmup):
        fn()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.reps
    print(json.dumps({"workload": name, "nnz": A.nnz, "T": m.T, "N": a.N, "kernel": a.kernel,
                      "form": a.form, "H": a.H, "W": a.W, "mode": a.mode, "chunks": grid,
                      "ms": ms, "wall_s": time.perf_counter() - t0,
                      "device_status": metcf.device_status(clear=True)}), flush=True)


if __name__ == "__main__":
    main()
