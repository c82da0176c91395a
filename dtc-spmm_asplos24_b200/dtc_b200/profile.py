"""Runs one SpMM configuration a few times: a fixed target for profilers.

    python -m dtc_b200.profile --scale 19 --form bf16x2x3 --H 32 --mode 0 --reps 3

Builds the seeded R-MAT(0.57, 0.19, 0.19, 0.05) matrix of 2^scale nodes
(symmetrised, self-loops, GCN values; --stencil 126 for the 27-point stencil
instead), converts it to ME-TCF of block shape H x W, packs a seeded N(0,1)
B into the form's storage, runs --warmup untimed products and --reps timed
ones, and prints one JSON line with the mean CUDA-event time per product.
With --kernel pack or --kernel convert it repeats the B pack or the ME-TCF
conversion instead; the kernels around the product repeat with tca (the TCA
permutation of the matrix), permute (P A P^T under a seeded permutation),
transpose (A^T), coo (CSR rebuild from the matrix's shuffled edge list),
features (the 48 schedule features) and mlp (one training step of the
48-64-64-432 schedule network on a batch of --batch feature rows, then its
argmin choice). Modes that do not read the ME-TCF arrays do not build them, so
only the mode's own kernels run after setup and a profiler's kernel filter
(for example ``ncu -k regex:k_spmm -c 1``) lands on the product.
"""
import argparse
import json
import time

import numpy as np
import torch

from . import costmodel, dataset, gen, metcf, reorder, tune
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
    ap.add_argument("--kernel", default="spmm",
                    choices=["spmm", "pack", "convert", "tca", "permute", "transpose", "coo",
                             "features", "mlp"])
    ap.add_argument("--batch", type=int, default=1024, help="feature rows per MLP step")
    a = ap.parse_args(argv)
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    if a.kernel == "mlp":
        return _mlp(a, dev)
    if a.stencil:
        A = gen.stencil27(a.stencil, seed=0)
        name = f"stencil27-{a.stencil}^3"
    else:
        A = gen.rmat(a.scale, 16.0, 0.57, 0.19, 0.19, seed=0)
        name = f"rmat-2^{a.scale}-sym-gcn"
    rp = torch.from_numpy(A.rowptr).to(dev)
    col = torch.from_numpy(A.col).to(dev)
    val = torch.from_numpy(A.val).to(dev)
    if a.kernel in ("tca", "permute", "transpose", "coo"):
        return _relabel(a, dev, A, name, rp, col, val)
    if a.kernel == "features":  # the schedule features are defined on the 16 x 8 ME-TCF
        a.H, a.W = 16, 8
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
    elif a.kernel == "features":
        fn = lambda: costmodel.features(rp, col, m, a.N)
    else:
        fn = lambda: metcf.convert(rp, col, A.M, H=a.H, W=a.W, values=val, device=dev)
    ms, wall = _time(fn, a.warmup, a.reps)
    print(json.dumps({"workload": name, "nnz": A.nnz, "T": m.T, "N": a.N, "kernel": a.kernel,
                      "form": a.form, "H": a.H, "W": a.W, "mode": a.mode, "chunks": grid,
                      "ms": ms, "wall_s": wall,
                      "device_status": metcf.device_status(clear=True)}), flush=True)


def _time(fn, warmup, reps):
    """Mean CUDA-event time (ms) of reps calls after warmup calls, and wall seconds."""
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / max(reps, 1), time.perf_counter() - t0


def _relabel(a, dev, A, name, rp, col, val):
    if a.kernel == "tca":
        fn = lambda: reorder.tca_perm(rp, col, A.M)
    elif a.kernel == "permute":
        g = torch.Generator(device="cpu").manual_seed(0)
        perm = torch.randperm(A.M, generator=g).to(dev, torch.int32)
        fn = lambda: metcf.permute_csr(rp, col, val, perm)
    elif a.kernel == "transpose":
        fn = lambda: metcf.transpose_csr(rp, col, val, A.K)
    else:
        rng = np.random.default_rng(0)
        order = rng.permutation(A.nnz)
        src = np.repeat(np.arange(A.M, dtype=np.int32), np.diff(A.rowptr))[order]
        s_d = torch.from_numpy(src).to(dev)
        d_d = torch.from_numpy(np.ascontiguousarray(A.col[order])).to(dev)
        fn = lambda: dataset.coo_to_csr(s_d, d_d, A.M, A.K, device=dev)
    ms, wall = _time(fn, a.warmup, a.reps)
    print(json.dumps({"workload": name, "nnz": A.nnz, "kernel": a.kernel, "ms": ms,
                      "wall_s": wall, "device_status": metcf.device_status(clear=True)}),
          flush=True)


def _mlp(a, dev):
    rng = np.random.default_rng(0)
    net = costmodel.MLP(device=dev)
    X = torch.from_numpy(rng.standard_normal((a.batch, costmodel.NFEAT)).astype(np.float32)).to(dev)
    T = torch.from_numpy(rng.random((a.batch, costmodel.K)).astype(np.float32)).to(dev)
    Mk = torch.ones_like(T)
    feas = np.ones(costmodel.K, np.uint8)

    def fn():
        net.train(X, T, Mk, steps=1)
        net.choose(X, feas)
    ms, wall = _time(fn, a.warmup, a.reps)
    print(json.dumps({"kernel": "mlp", "batch": a.batch, "dims": list(net.dims), "ms": ms,
                      "wall_s": wall, "device_status": metcf.device_status(clear=True)}),
          flush=True)


if __name__ == "__main__":
    main()
