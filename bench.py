"""Benchmark of the B200-native DTC-SpMM path.

Workload (default): power-law graph SpMM -- R-MAT(0.57, 0.19, 0.19, 0.05),
2^20 nodes, 16 * 2^20 generated edges, symmetrised + self-loops + duplicates
removed, GCN-normalised values; B = 2^20 x 128 fp32 N(0,1); seeded synthetic
data standing in for the reference's graph datasets.

One step = one SpMM C = A * B over the whole matrix with A's ME-TCF arrays and
B already resident in HBM (`value`, GFLOP/s = 2 * nnz * N / t), in the form
and schedule the learned cost model picks among the forms within 1e-5
relative error (window height, mode, waves, N-tiles, B storage form, TCA
reorder; `dtype` names the form it picked). Beside it: the plain TF32 drop-in
with its autotuned schedule (the speed-up reference), the exhaustive
autotuner's best split schedule, fixed schedules of every B form, the B pack
and ME-TCF conversion times, and the host CSR SpMM. `e2e` streams products
through dtc_b200.hostpipe.HostPipeline: pinned host B in, pack, SpMM, C back to
pinned host memory, with the copies of consecutive products overlapped.

  python bench.py [--gpus N --steps K --warmup W]     # this library
  python bench.py --impl reference                    # the reference's own kernels

The reference arm runs the unmodified reference extension rebuilt for sm_100a
(oracle/_ref, built from the reference sources by oracle/build_ref.py) through
its own API: preprocess_gpu, then run_DTCSpMM_balance with "float4_split",
the plan the reference's schedule table gives power-law graphs at N = 128
(scripts/DTCSpMM/run_DTC_SpMM.py:16). Each of its calls runs 1000 launches
(DTC-SpMM/DTCSpMM_kernel.cu:18); one step is one call, its time per product is
the call's time / 1000. Without the built reference the arm falls back to the
host CSR SpMM port and says so.

Multi-GPU (torchrun): every rank runs its own replica of the workload (row
windows are independent; there is no data-path collective); timing is the
max over ranks, `value` the sum of the ranks' work over that time.
"""
import argparse
import contextlib
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "dtc-spmm_asplos24_b200")
sys.path.insert(0, PKG)
sys.path.insert(0, ROOT)

METRIC = "SpMM GFLOP/s (2·nnz·N) & HBM-roofline %: tuned vs plain TF32 at ≤1e-5 rel err"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
MIN_TIMED_S = 1.0  # the timed region repeats its K steps until it lasts this long
REF_LAUNCHES = 1000  # launches per reference SpMM call (DTC-SpMM/DTCSpMM_kernel.cu:18)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


def make_workload(args):
    from dtc_b200 import gen
    if args.config == "rmat":
        A = gen.rmat(args.scale, 16.0, 0.57, 0.19, 0.19, seed=0)
        N = args.N or 128
        name = f"rmat-2^{args.scale}-sym-gcn-N{N}"
    elif args.config == "stencil":
        A = gen.stencil27(126, seed=0)
        N = args.N or 256
        name = f"stencil27-126^3-N{N}"
    else:
        A = gen.uniform(4096, mean=8.0, seed=0)
        N = args.N or 32
        name = f"uniform-4096-poisson8-N{N}"
    B = gen.normal(A.K, N, seed=1)
    return A, B, N, name


TRAFFIC_FILES = {"rmat-2^20-sym-gcn-N128": "dram_traffic_rmat20_N128.md"}


def measured_traffic(workload, kernel):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of
    `kernel` on `workload` from the committed ncu summary, or None."""
    f = TRAFFIC_FILES.get(workload)
    p = os.path.join(ROOT, "profiles", f) if f else None
    if not p or not os.path.exists(p):
        return None
    for line in open(p):
        cells = [x.strip().strip("`") for x in line.strip().strip("|").split("|")]
        if len(cells) >= 2 and cells[0] == kernel and cells[1].replace(",", "").isdigit():
            return int(cells[1].replace(",", ""))
    return None


def algorithmic_bytes(m, N, b_elem_bytes, with_values=True):
    """ME-TCF structure + gathered B rows (distinct per window) + C write."""
    T, nnz = m.T, m.nnz
    s2x = m.SparseAToX.view(T, m.W)
    valid = (s2x != 0)
    valid[:, 0] = True
    U = int(valid.sum().item())
    S = nnz * (1 + (4 if with_values else 0)) + 8 * T * 4 + (T + 1) * 4 + (m.nwin + 1) * 4
    return S + U * N * b_elem_bytes + m.M * N * 4, U, S


# --------------------------------------------------------------------- clocks
_REASONS = [("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
            ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
            ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
            ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
            ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown")]


class Clocks:
    """SM clock and clock-event reasons sampled through NVML every `period`
    seconds on a background thread while the timed region runs (nvidia-smi
    polling as the fallback)."""

    def __init__(self, device, period=0.005):
        self.device, self.period = device, period
        self.samples, self.max_mhz = [], None
        self._stop = threading.Event()
        self._thr = self._smi = None

    def _handle(self, nv):
        import torch
        pr = torch.cuda.get_device_properties(self.device)
        try:
            return nv.nvmlDeviceGetHandleByPciBusId(
                f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0")
        except Exception:
            return nv.nvmlDeviceGetHandleByUUID("GPU-" + str(pr.uuid))

    def _run(self, nv, h):
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((mhz, rs))
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self._nv = nv
            self._thr = threading.Thread(target=self._run, args=(nv, h), daemon=True)
            self._thr.start()
        except Exception:
            self._start_smi()
        time.sleep(0.05)
        return self

    def _start_smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        self._smi_path = os.path.join(tempfile.gettempdir(), f"dtc_clocks_{os.getpid()}.csv")
        try:
            self._smi = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device.index or 0}", f"--query-gpu={q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=open(self._smi_path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self._smi = None

    def __exit__(self, *a):
        self._stop.set()
        if self._thr:
            self._thr.join()
        if self._smi:
            self._smi.terminate()
            self._smi.wait()
            self._read_smi()

    def _read_smi(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self._smi_path).read().strip().splitlines():
            r = [x.strip() for x in line.split(",")]
            if len(r) < 6 or not r[0].isdigit():
                continue
            self.max_mhz = float(r[1])
            self.samples.append((float(r[0]), {n for n, v in zip(names, r[2:6]) if v == "Active"}))

    def summary(self):
        if not self.samples:
            return None
        reasons = set()
        for _, rs in self.samples:
            if isinstance(rs, set):
                reasons |= rs
            else:
                reasons |= {n for n, c in _REASONS
                            if hasattr(self._nv, c) and rs & getattr(self._nv, c)}
        sm = [s[0] for s in self.samples]
        return {"sm_mhz": float(np.median(sm)), "sm_min_mhz": float(min(sm)),
                "sm_max_mhz": float(self.max_mhz) if self.max_mhz else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml" if self._thr else "nvidia-smi"}


# ------------------------------------------------------------------ CPU parts
def cpu_baseline(A, B, N, budget_s=15.0):
    """Host FP32 CSR SpMM (the oracle's OpenMP port) on all host cores.

    Bounded sample: the full matrix, repeated while the budget lasts (at least
    twice, at most 10 times); the median run is reported.
    """
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    C = np.empty((A.M, N), np.float32)
    O.spmm_f32(A.rowptr, A.col, A.val, A.M, B, nthreads=cores, out=C)  # warm-up
    times = []
    t_end = time.perf_counter() + budget_s
    while len(times) < 2 or (time.perf_counter() < t_end and len(times) < 10):
        t0 = time.perf_counter()
        O.spmm_f32(A.rowptr, A.col, A.val, A.M, B, nthreads=cores, out=C)
        times.append(time.perf_counter() - t0)
    t = float(np.median(times))
    return {"value": 2.0 * A.nnz * N / t / 1e9, "unit": "GFLOP/s", "cores": cores,
            "kind": "port",
            "sample": f"full matrix ({A.nnz} nnz x N={N}), median of {len(times)} runs",
            "cpu_model": _cpu_model()}


def accuracy_vs_fp64(A, B, N, gpu_C, rows_per=64):
    """Relative Frobenius and max-abs error of the GPU result vs the FP64
    oracle on every `rows_per`-th row window (16 rows each)."""
    from oracle import oracle as O
    wins = np.arange(0, (A.M + 15) // 16, rows_per)
    rows = np.concatenate([np.arange(w * 16, min(w * 16 + 16, A.M)) for w in wins])
    lens = A.rowptr[rows + 1] - A.rowptr[rows]
    rp = np.zeros(len(rows) + 1, np.int64)
    rp[1:] = np.cumsum(lens)
    idx = np.concatenate([np.arange(A.rowptr[r], A.rowptr[r + 1]) for r in rows])
    C64 = O.spmm_f64(rp.astype(np.int32), A.col[idx], A.val[idx], len(rows), B)
    G = gpu_C[rows].astype(np.float64)
    return {"rel_fro": float(np.linalg.norm(G - C64) / np.linalg.norm(C64)),
            "max_abs": float(np.abs(G - C64).max()), "rows_checked": int(len(rows))}


def _cpu_model():
    try:
        for l in open("/proc/cpuinfo"):
            if l.startswith("model name"):
                return l.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ------------------------------------------------------------- reference arm
REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def _load_reference():
    """The reference extension rebuilt for sm_100a, or None when absent."""
    import glob
    import torch
    if not glob.glob(os.path.join(REF_DIR, "DTCSpMM*.so")) or not torch.cuda.is_available():
        return None
    sys.path.insert(0, REF_DIR)
    import DTCSpMM as ref
    assert os.path.dirname(os.path.abspath(ref.__file__)) == REF_DIR, ref.__file__
    return ref


@contextlib.contextmanager
def _quiet_cwd():
    """The reference prints progress to stdout and appends a CSV row to its
    working directory: run it in a scratch directory with stdout sent to stderr,
    so the arm's stdout carries only its JSON line."""
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(2, 1)
    old = os.getcwd()
    with tempfile.TemporaryDirectory() as d:
        os.chdir(d)
        try:
            yield
        finally:
            os.chdir(old)
            sys.stdout.flush()
            os.dup2(saved, 1)
            os.close(saved)


def run_reference_arm(args, rank, world):
    """The reference's own path on this GPU (rank 0 only, N = 1 workload)."""
    if rank != 0:
        return
    A, Bh, N, name = make_workload(args)
    flops = 2.0 * A.nnz * N
    cpu = cpu_baseline(A, Bh, N, budget_s=10.0)
    ref = _load_reference()
    base = {"impl": "reference", "metric": METRIC, "unit": "GFLOP/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "data": "synthetic",
            "config": {"workload": name, "nnz": A.nnz, "num_nodes": A.M, "N": N}}
    if ref is None:
        v = cpu["value"]
        line = dict(base, value=v, ms_per_step=flops / v / 1e6, dtype="f32",
                    note="reference extension (oracle/_ref) or GPU absent: host CSR SpMM port",
                    cpu_baseline=cpu, e2e={"value": v, "unit": "GFLOP/s",
                                           "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(line), flush=True)
        return
    import torch
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    col = torch.from_numpy(A.col).to(dev)
    rp = torch.from_numpy(A.rowptr).to(dev)
    nwin = (A.M + 15) // 16

    def preprocess():
        bp = torch.zeros(nwin, dtype=torch.int32, device=dev)
        e2c = torch.zeros(A.nnz, dtype=torch.int32, device=dev)
        e2r = torch.zeros(A.nnz, dtype=torch.int32, device=dev)
        with _quiet_cwd():
            r = ref.preprocess_gpu(col, rp, A.M, 16, 8, bp, e2c, e2r)
        torch.cuda.synchronize()
        return r

    conv = []
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rwo, rowid, tile, toff, s2x, T = preprocess()
        conv.append((time.perf_counter() - t0) * 1e3)
    X = torch.from_numpy(Bh).to(dev)
    plan = "float4_split"

    def call():
        with _quiet_cwd():
            return ref.run_DTCSpMM_balance(X, rowid, tile, toff, s2x, A.M, plan)[0]

    for _ in range(args.warmup):
        Cr = call()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(args.steps)]
    with Clocks(dev) as clk:
        for a, b in evs:
            a.record()
            Cr = call()
            b.record()
        torch.cuda.synchronize()
    per_call = [a.elapsed_time(b) for a, b in evs]
    ms = float(np.mean(per_call)) / REF_LAUNCHES
    # e2e: the reference's API takes and returns device tensors; a host caller
    # adds one pinned H2D copy of B and one D2H copy of C per product
    Bpin = torch.from_numpy(Bh).pin_memory()
    Cpin = torch.empty((A.M, N), dtype=torch.float32).pin_memory()
    h2d, d2h = [], []
    for _ in range(5):
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        e[0].record()
        X.copy_(Bpin, non_blocking=True)
        e[1].record()
        Cpin.copy_(Cr, non_blocking=True)
        e[2].record()
        torch.cuda.synchronize()
        h2d.append(e[0].elapsed_time(e[1]))
        d2h.append(e[1].elapsed_time(e[2]))
    e2e_ms = float(np.median(h2d)) + ms + float(np.median(d2h))
    v = flops / (ms * 1e-3) / 1e9
    line = dict(base, value=v, ms_per_step=ms, dtype="tf32 (fp32 B, TF32 mma.sync, A = 1)",
                kernel=f"run_DTCSpMM_balance('{plan}') rebuilt for sm_100a",
                ms_per_call=float(np.mean(per_call)), launches_per_call=REF_LAUNCHES,
                convert_ms=float(np.median(conv)), T=int(T),
                clocks=clk.summary(), cpu_baseline=cpu,
                e2e={"value": flops / (e2e_ms * 1e-3) / 1e9, "unit": "GFLOP/s",
                     "h2d_bytes_per_step": int(Bh.nbytes), "d2h_bytes_per_step": int(A.M * N * 4),
                     "ms": e2e_ms, "h2d_ms": float(np.median(h2d)),
                     "d2h_ms": float(np.median(d2h)),
                     "how": "pinned H2D of B + one product (call / 1000) + D2H of C, serial"})
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------- batched
def run_batched(args):
    """Batched uneven matrices: one graph-captured launch over the stacked batch
    vs one window-scheduled launch per matrix (the reference-style loop)."""
    import torch
    from dtc_b200 import batched
    torch.cuda.set_device(0)
    N = args.N or 64
    t0 = time.perf_counter()
    mats, Bs = batched.zipf_batch(count=args.batch, N=N, seed=0)
    gen_s = time.perf_counter() - t0
    nnz = sum(m.nnz for m in mats)
    flops = 2.0 * nnz * N
    Bt = [torch.from_numpy(b).cuda() for b in Bs]

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    bs = batched.BatchedSpMM(mats, N)
    bs.load(Bt)
    t0 = time.perf_counter()
    table = bs.autotune(reps=3)
    tune_s = time.perf_counter() - t0
    bs.capture()
    one_ms = timed(bs.run, args.steps, args.warmup)
    # the same launch with one CTA per chunk (hardware block scheduler, no queue)
    bs.queue = False
    bs._alloc_ws()
    bs.capture()
    static_ms = timed(bs.run, args.steps, args.warmup)
    ms_sep, run_sep = batched.separate_launches(mats, N)
    outs = [torch.empty((m.M, N), device="cuda") for m in mats]
    sep_ms = timed(lambda: run_sep(Bt, outs), max(3, args.steps // 4), 2)
    g_sep = batched.separate_launches_graph(ms_sep, Bt, outs)
    sep_graph_ms = timed(g_sep.replay, max(3, args.steps // 4), 2)
    line = {"metric": "batched SpMM GFLOP/s (2*nnz*N), one graph launch vs per-matrix launches",
            "value": flops / (one_ms * 1e-3) / 1e9, "unit": "GFLOP/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": one_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "tf32",
            "data": "synthetic",
            "config": {"workload": f"{args.batch} zipf(2.1) matrices, rows log-uniform "
                                   f"[256, 65536], N={N}", "nnz": int(nnz),
                       "rows": int(sum(m.M for m in mats)), "T": bs.m.T},
            "one_cta_per_chunk_ms": static_ms,
            "separate_launches_ms": sep_ms,
            "separate_launches_gflops": flops / (sep_ms * 1e-3) / 1e9,
            "separate_launches_one_graph_ms": sep_graph_ms,
            "speedup_vs_separate": sep_ms / one_ms,
            "speedup_vs_separate_one_graph": sep_graph_ms / one_ms,
            "speedup_vs_one_cta_per_chunk": static_ms / one_ms,
            "gpu_launches": (3 if bs.mode == 1 and bs.grid > 1 else 2) * args.steps,
            "schedule": {"H": bs.m.H, "mode": bs.mode, "grid": bs.grid, "ntile": bs.ntile,
                         "autotune_ms": {h: v.ms for h, v in table.items()},
                         "autotune_s": tune_s},
            "generation_s": gen_s}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------- balance report
def run_balance_report(args):
    """Per-CTA busy times (dtc_set_cta_timer) of one SpMM launch per schedule:
    window mode vs strict balance, persistent CTAs on the chunk queue vs one
    CTA per chunk; plain TF32 and the BF16X2 split form at window height 32."""
    import torch
    from dtc_b200 import balance, metcf, tune, B_F32, B_BF16X2, PREC_TF32, PREC_SPLIT3
    torch.cuda.set_device(0)
    A, Bh, N, name = make_workload(args)
    dev = torch.device("cuda", 0)
    B = torch.from_numpy(Bh).to(dev)
    m = metcf.convert(A.rowptr, A.col, A.M, H=32, values=A.val, device=dev)
    out = torch.empty((A.M, N), device=dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    rows = {}
    for form, fmt, prec in (("tf32", B_F32, PREC_TF32), ("bf16x2x3", B_BF16X2, PREC_SPLIT3)):
        planes = [B] if fmt == B_F32 else metcf.pack_b(B, fmt)
        for mode in (0, 1):
            grid = min(16 * sms, m.T)
            full = metcf.spmm_ex_workspace_bytes(m, N, mode, grid)
            for queue in (True, False):
                wsb = full if queue else max(full - _queue_bytes(m, grid), 0)
                ws = torch.empty(max(wsb, 1), dtype=torch.uint8, device=dev)
                fn = lambda: metcf.spmm_ex(m, planes, fmt, N, prec, mode=mode, grid=grid,
                                           out=out, workspace=ws if wsb else None)
                for _ in range(3):
                    fn()
                r = balance.cta_report(fn, capacity=max(grid, sms) + 8, device=dev)
                rows[f"{form}_h32_mode{mode}_{'persistent' if queue else 'one-cta-per-chunk'}"] = r
    line = {"metric": "per-CTA busy time of one SpMM launch (us)", "workload": name,
            "nnz": A.nnz, "T": m.T, "chunks": min(16 * sms, m.T), "schedules": rows}
    print(json.dumps(line), flush=True)


def _queue_bytes(m, grid):
    """Bytes of the chunk-queue region spmm_ex_workspace_bytes includes."""
    from dtc_b200 import metcf
    return metcf.spmm_ex_workspace_bytes(m, 128, 0, grid)


# ------------------------------------------------------------------ our arm
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="rmat",
                    choices=["rmat", "stencil", "uniform", "batched", "balance"])
    ap.add_argument("--batch", type=int, default=512)
    ap.add_argument("--scale", type=int, default=20)
    ap.add_argument("--N", type=int, default=0)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.config == "batched":
        return run_batched(args)
    if args.config == "balance":
        args.config = "rmat"
        return run_balance_report(args)

    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from dtc_b200 import (metcf, replicas, hostpipe, B_F32, B_SPLIT24, B_BF16, B_FP8, B_BF16X2,
                          PREC_TF32, PREC_SPLIT3, PREC_SPLIT4)

    A, Bh, N, name = make_workload(args)
    dev = torch.device("cuda", local)
    m = metcf.convert(A.rowptr, A.col, A.M, values=A.val, device=dev)
    B = torch.from_numpy(Bh).to(dev)
    flops = 2.0 * A.nnz * N
    peaks, peak_kind = load_peaks()

    planes = {B_SPLIT24: metcf.pack_b(B, B_SPLIT24), B_BF16: metcf.pack_b(B, B_BF16),
              B_BF16X2: metcf.pack_b(B, B_BF16X2),
              B_FP8: metcf.pack_b(B, B_FP8)}
    outs = {}

    def out_for(k):
        if k not in outs:
            outs[k] = torch.empty((A.M, N), dtype=torch.float32, device=dev)
        return outs[k]

    wsb = max(metcf.spmm_balance_workspace_bytes(m, N), 1)
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)

    def ex(fmt, prec, mode, k):
        pl = [B] if fmt == B_F32 else planes[fmt]
        return lambda: metcf.spmm_ex(m, pl, fmt, N, prec, mode=mode, out=out_for(k),
                                     workspace=ws)

    # (storage form, precision, schedule) -> bytes per gathered B element
    forms = {
        "tf32_window": (ex(B_F32, PREC_TF32, 0, "tf32_window"), 4.0),
        "tf32_balance": (ex(B_F32, PREC_TF32, 1, "tf32_balance"), 4.0),
        "split24x4_window": (ex(B_SPLIT24, PREC_SPLIT4, 0, "split24x4_window"), 3.0),
        "split24x4_balance": (ex(B_SPLIT24, PREC_SPLIT4, 1, "split24x4_balance"), 3.0),
        "split24x3_balance": (ex(B_SPLIT24, PREC_SPLIT3, 1, "split24x3_balance"), 3.0),
        "bf16x2x3_balance": (ex(B_BF16X2, PREC_SPLIT3, 1, "bf16x2x3_balance"), 4.0),
        "bf16_balance": (ex(B_BF16, PREC_SPLIT4, 1, "bf16_balance"), 2.0),
        "fp8_balance": (ex(B_FP8, PREC_SPLIT4, 1, "fp8_balance"), 1.0 + 4.0 / N),
    }

    def timed(fn, steps, warmup, min_s=0.0, stream=None):
        """Times `steps` calls of fn between CUDA events on the launching stream,
        after `warmup` untimed calls and a barrier + synchronize. The K-step block
        repeats until the region lasts `min_s`; returns (mean ms per step over all
        blocks, max over ranks; per-step event times; blocks)."""
        for _ in range(warmup):
            fn()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        st = stream or torch.cuda.current_stream()
        per, total, blocks = [], 0.0, 0
        while True:
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(steps)]
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            for a, b in evs:
                a.record(st)
                fn()
                b.record(st)
            e1.record(st)
            torch.cuda.synchronize()
            per += [a.elapsed_time(b) for a, b in evs]
            total += e0.elapsed_time(e1)
            blocks += 1
            # every rank runs the same number of blocks
            more = torch.tensor([1.0 if total < min_s * 1e3 else 0.0], device=dev)
            if dist:
                dist.all_reduce(more, op=dist.ReduceOp.MAX)
            if more.item() == 0.0:
                break
        tmax = replicas.max_over_ranks(float(total), dist, dev)
        return tmax / (steps * blocks), per, blocks

    results = {}
    for k, (fn, eb) in forms.items():
        ms, per, _ = timed(fn, max(3, args.steps // 2), args.warmup)
        nbytes = algorithmic_bytes(m, N, eb)[0]
        results[k] = {"ms": ms, "gflops": flops / (ms * 1e-3) / 1e9,
                      "hbm_frac": nbytes / (float(np.mean(per)) * 1e-3) / 1e9 / peaks["hbm_gbs"],
                      "bytes_per_B_elem": eb}
    # autotuned schedules: every (mode, chunks, N-tile) at block shapes 16 x 8, 32 x 8 and
    # 16 x 16 for the plain TF32 drop-in and for the two B forms within 1e-5 (dtc_autotune)
    from dtc_b200 import tune, costmodel, reorder as reorder_mod
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    mets = {(16, 8): m,
            (32, 8): metcf.convert(A.rowptr, A.col, A.M, H=32, values=A.val, device=dev),
            (16, 16): metcf.convert(A.rowptr, A.col, A.M, H=16, W=16, values=A.val, device=dev)}
    tuned_tbl = {}
    for H, mm in mets.items():
        ws_t = tune.workspace_for(mm, N, dev)
        for fo in ("tf32", "split24x4", "split24x3", "bf16x2x3"):
            fmt, prec = tune.FORMS[fo][0], tune.FORMS[fo][1]
            pl = [B] if fo == "tf32" else planes[fmt]
            scheds, best = tune.autotune(mm, pl, fmt, N, prec, reps=3, out=out_for("tune"),
                                         workspace=ws_t)
            tuned_tbl[(fo, H)] = best
        del ws_t
    plain_key = min((k for k in tuned_tbl if k[0] == "tf32"), key=lambda k: tuned_tbl[k].ms)
    shape_name = lambda hw: f"h{hw[0]}w{hw[1]}"
    exh_key = min((k for k in tuned_tbl if k[0] != "tf32"), key=lambda k: tuned_tbl[k].ms)

    # the learned scheduler's choice (features -> MLP on the GPU, its 8 cheapest
    # predicted classes timed on this matrix); the exhaustive autotuner is its
    # fallback when no weights match the class space
    t0 = time.perf_counter()
    plan = costmodel.Scheduler(device=dev).plan(torch.from_numpy(A.rowptr).to(dev),
                                                torch.from_numpy(A.col).to(dev), m, N, B=B,
                                                verify_top=8)
    plan_s = time.perf_counter() - t0
    perm = None
    At = A
    if plan.reorder:
        t0 = time.perf_counter()
        perm, rp2, c2, v2 = reorder_mod.reorder(torch.from_numpy(A.rowptr).to(dev),
                                                torch.from_numpy(A.col).to(dev),
                                                torch.from_numpy(A.val).to(dev), A.M)
        torch.cuda.synchronize()
        tca_s = time.perf_counter() - t0
        mt = metcf.convert(rp2, c2, A.M, H=plan.H, W=getattr(plan, "W", 8), values=v2,
                           device=dev)
        At = type("CSR", (), dict(rowptr=rp2.cpu().numpy(), col=c2.cpu().numpy(),
                                  val=v2.cpu().numpy(), M=A.M, K=A.K, nnz=A.nnz))
        Bt = B.index_select(0, perm.long()).contiguous()
    else:
        tca_s = 0.0
        mt = mets[(plan.H, getattr(plan, "W", 8))]
        Bt = B
    fmt_t, prec_t, eb_t = tune.FORMS[plan.form][0], tune.FORMS[plan.form][1], \
        tune.FORMS[plan.form][2]
    planes_t = [Bt] if fmt_t == B_F32 else metcf.pack_b(Bt, fmt_t)
    sched = tune.Schedule(mode=plan.mode, waves=plan.waves, ntile=plan.ntile,
                          grid=min(plan.waves * sms, max(mt.T, 1)), ms=0.0)
    ws_m = tune.workspace_for(mt, N, dev)
    out_t = out_for("tuned")
    tuned_fn = lambda: tune.run(mt, planes_t, fmt_t, N, prec_t, sched, out=out_t, workspace=ws_m)
    tuned = f"{plan.form}_{shape_name((mt.H, mt.W))}_mode{plan.mode}_w{plan.waves}" + \
        f"_nt{plan.ntile}" + ("_tca" if plan.reorder else "")
    launches = metcf.spmm_ex_launches(mt, sched.mode, sched.grid)

    # the plain TF32 drop-in at its autotuned schedule, timed like the headline
    mp = mets[plain_key[1]]
    sp = tuned_tbl[plain_key]
    ws_p = tune.workspace_for(mp, N, dev)
    plain_fn = lambda: tune.run(mp, [B], B_F32, N, PREC_TF32, sp, out=out_for("plain"),
                                workspace=ws_p)
    plain_ms, plain_per, _ = timed(plain_fn, args.steps, args.warmup, MIN_TIMED_S)

    # headline timed region: K steps of the model-scheduled form (repeated until
    # it lasts MIN_TIMED_S), clocks sampled during it
    with Clocks(dev) as clk:
        ms, per, blocks = timed(tuned_fn, args.steps, args.warmup, MIN_TIMED_S)
    clocks = clk.summary()
    value = replicas.aggregate_gflops(flops, ms, world)

    # the B pack (fp32 -> storage form) and the ME-TCF conversion, timed alone
    pack_ms = 0.0
    if fmt_t != B_F32:
        pack_ms, _, _ = timed(lambda: metcf.pack_b_into(Bt, fmt_t, planes_t), 10, 3)
    # (CSR already on the device, like the reference's preprocess_gpu inputs)
    conv = []
    rp_t, col_t, val_t = (torch.from_numpy(np.ascontiguousarray(x)).to(dev)
                          for x in (At.rowptr, At.col, At.val))
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        metcf.convert(rp_t, col_t, A.M, H=mt.H, W=mt.W, values=val_t, device=dev)
        torch.cuda.synchronize()
        conv.append((time.perf_counter() - t0) * 1e3)
    conv16 = []
    rp_d, col_d = torch.from_numpy(A.rowptr).to(dev), torch.from_numpy(A.col).to(dev)
    for _ in range(3):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        metcf.convert(rp_d, col_d, A.M, H=16, device=dev)
        torch.cuda.synchronize()
        conv16.append((time.perf_counter() - t0) * 1e3)

    nbytes, U, S = algorithmic_bytes(mt, N, eb_t)
    kern_ms = float(np.mean(per))
    achieved = nbytes / (kern_ms * 1e-3) / 1e9
    traffic = measured_traffic(name, tuned)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                "dram_frac": (traffic / (kern_ms * 1e-3) / 1e9 / peaks["hbm_gbs"]
                              if traffic else None),
                "peak_kind": peak_kind, "algorithmic_bytes": nbytes, "distinct_rows_U": U,
                "metcf_bytes": S, "compulsory_bytes": S + A.K * N * eb_t + A.M * N * 4,
                "kernel": tuned, "kernel_ms": kern_ms,
                "note": "achieved = algorithmic bytes (ME-TCF + distinct gathered B rows + C) / "
                        "mean step time; dram_frac = measured DRAM bytes / the same time"}

    # end to end through the public API with host buffers: pinned fp32 B ->
    # device (row gather when reordered) -> storage-form pack -> SpMM -> pinned
    # host C, consecutive products overlapped on three streams
    Bpin = torch.from_numpy(Bh).pin_memory()
    Cpin = torch.empty((A.M, N), dtype=torch.float32).pin_memory()
    pipe = hostpipe.HostPipeline(mt, N, fmt_t, prec_t, mode=sched.mode, grid=sched.grid,
                                 ntile=sched.ntile, perm=perm)
    for _ in range(2):
        pipe.submit(Bpin, Cpin)
    pipe.synchronize()
    torch.cuda.synchronize()
    e2e_steps = max(4, args.steps)
    s_in, _, s_out = pipe.streams
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    e0.record(s_in)
    for _ in range(e2e_steps):
        pipe.submit(Bpin, Cpin)
    e1.record(s_out)
    torch.cuda.synchronize()
    e_ms = replicas.max_over_ranks(float(e0.elapsed_time(e1)), dist, dev) / e2e_steps
    e2e = {"value": world * flops / (e_ms * 1e-3) / 1e9, "unit": "GFLOP/s", "ms": e_ms,
           "h2d_bytes_per_step": int(Bh.nbytes), "d2h_bytes_per_step": int(A.M * N * 4),
           "steps": e2e_steps, "api": "dtc_b200.hostpipe.HostPipeline (pack_b + spmm_ex)"}
    learned = {"class": costmodel.CLASSES[plan.cls], "source": plan.source,
               "plan_s": plan_s, "tca_reorder_s": tca_s, "T": mt.T, "ms": kern_ms,
               "exhaustive_no_reorder": {"form": exh_key[0], "shape": shape_name(exh_key[1]),
                                         "mode": tuned_tbl[exh_key].mode,
                                         "waves": tuned_tbl[exh_key].waves,
                                         "ntile": tuned_tbl[exh_key].ntile,
                                         "ms": tuned_tbl[exh_key].ms},
               "plain_tf32_tuned": {"shape": shape_name(plain_key[1]), "mode": sp.mode,
                                    "waves": sp.waves,
                                    "ntile": sp.ntile, "ms": plain_ms,
                                    "autotune_ms": tuned_tbl[plain_key].ms},
               "autotune": {f"{k[0]}_{shape_name(k[1])}": v.ms for k, v in tuned_tbl.items()}}
    tf32_best = min(("tf32_window", "tf32_balance"), key=lambda k: results[k]["ms"])

    cpu, errs = (None, {})
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(A, Bh, N)
        for k in (tf32_best, "split24x3_balance", "bf16x2x3_balance", "bf16_balance",
                  "fp8_balance"):
            forms[k][0]()
            torch.cuda.synchronize()
            errs[k] = accuracy_vs_fp64(A, Bh, N, outs[k].cpu().numpy())
            results[k]["rel_err_vs_fp64"] = errs[k]["rel_fro"]
            results[k]["max_abs_err"] = errs[k]["max_abs"]
        tuned_fn()
        torch.cuda.synchronize()
        errs[tuned] = accuracy_vs_fp64(At, Bt.cpu().numpy(), N, out_t.cpu().numpy())
        errs["e2e"] = accuracy_vs_fp64(A, Bh, N, Cpin.numpy())

    if rank == 0:
        dtype = {"tf32": "tf32", "split24x4": "bf16 split, 4-term (SPLIT24 B), fp32 accumulate",
                 "split24x3": "bf16 split, 3-term (SPLIT24 B), fp32 accumulate",
                 "bf16x2x3": "bf16 split, 3-term (BF16X2 B), fp32 accumulate",
                 "bf16": "bf16", "fp8": "e4m3"}[plan.form]
        line = {"metric": METRIC, "value": value,
                "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": dtype, "data": "synthetic",
                "config": {"workload": name, "num_nodes": A.M, "nnz": A.nnz, "N": N,
                           "T": mt.T, "form": tuned,
                           "plain_form": f"tf32_{shape_name(plain_key[1])} (autotuned)",
                           "l2": "inputs larger than L2 (B %.0f MiB fp32, ME-TCF %.0f MB); no flush"
                           % (A.K * N * 4 / 2 ** 20, S / 1e6),
                           "timed_blocks": blocks,
                           "timed_region_ms": ms * args.steps * blocks},
                "hbm_roofline_frac": roofline["frac"],
                "speedup_vs_plain_tf32": plain_ms / ms,
                "pack_ms": pack_ms, "value_incl_pack": flops / ((ms + pack_ms) * 1e-3) / 1e9,
                "speedup_vs_plain_tf32_incl_pack": plain_ms / (ms + pack_ms),
                "convert_ms": float(np.median(conv)), "convert_h16_ms": float(np.median(conv16)),
                "forms": results, "learned_schedule": learned, "roofline": roofline,
                "e2e": e2e, "cpu_baseline": cpu, "accuracy_vs_fp64": errs.get(tuned),
                "accuracy_e2e_vs_fp64": errs.get("e2e"),
                "clocks": clocks,
                "gpu_launches": launches * args.steps * blocks}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
