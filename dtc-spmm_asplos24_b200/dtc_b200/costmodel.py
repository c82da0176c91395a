"""Learned schedule cost model: features (dtc_features) -> MLP 48 -> 64 -> 64 -> K
(dtc_mlp_* kernels) -> the schedule class with the lowest predicted cost.

The reference fixes its schedule by hand per dataset and N
(scripts/DTCSpMM/run_DTC_SpMM.py:10-30). Here a class is one full choice

    (window height, compaction width, mode, waves, N-tile, B form, reorder)

with TC blocks of 16 x 8, 32 x 8 or 16 x 16 (window height x compaction width;
the reference's blockSize_h x blockSize_w), mode 0 (window-scheduled) or 1
(strict balance), waves in {1,2,4,8,16,32,64} in window mode and {1,2,4,8,16}
in balance mode (chunks = waves x SMs, so the split threshold is ceil(T /
chunks) blocks), N-tiles per CTA in {1,2,4}, two B forms within 1e-5
relative error (SPLIT24, 3 bytes per element rebuilt on chip, and BF16X2, 4
bytes per element used as stored; both with 3-term products) and TCA reorder off or
on. The network predicts, for every class, log(t_class / t_best) of the SpMM
kernel; it is trained on timings the library measures itself on seeded
synthetic matrices (``collect``), entirely with the library's own CUDA kernels
(forward, backward, Adam). The model changes only which schedule runs: every
class computes the same product within its form's error bound. The exhaustive
autotuner (``tune.autotune`` over every class) is its fallback and the
reference point of its regret.
"""
import ctypes as C
import math
import os
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib, gen, metcf, reorder as reorder_mod, tune
from ._lib import MlpDims, call
from .metcf import _ptr, _stream

NFEAT = 48
SHAPES = ((16, 8), (32, 8), (16, 16))  # (window height, compaction width)
WAVES = {0: (1, 2, 4, 8, 16, 32, 64), 1: (1, 2, 4, 8, 16)}  # per mode
NTILES = (1, 2, 4)
FORMS = ("split24x3", "bf16x2x3")
CLASSES = [dict(H=h, W=w, mode=mo, waves=wv, ntile=nt, form=fo, reorder=ro)
           for ro in (0, 1) for h, w in SHAPES for fo in FORMS for mo in (0, 1) for wv in WAVES[mo]
           for nt in NTILES]
K = len(CLASSES)
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
DATASET_PATH = os.path.join(DATA_DIR, "costmodel_dataset.npz")
WEIGHTS_PATH = os.path.join(DATA_DIR, "costmodel_weights.npz")


def auto_ntile(N, H=16, W=8):
    """N-tiles per CTA the split kernels use when uncapped (2 at most at window
    height 32 or compaction width 16)."""
    nt = 1 if N <= 128 else 2 if N <= 256 else 4
    return min(nt, 2) if (H == 32 or W == 16) else nt


def feasible(N):
    """uint8 [K]: classes whose N-tile the kernels run for width N."""
    return np.array([c["ntile"] <= auto_ntile(N, c["H"], c["W"]) for c in CLASSES], np.uint8)


_INDEX = {(c["mode"], c["waves"], c["ntile"], c["form"], c["reorder"], c["H"], c["W"]): i
          for i, c in enumerate(CLASSES)}


def class_of(mode, waves, ntile, form, reorder, H=16, W=8):
    return _INDEX[(mode, waves, ntile, form, reorder, H, W)]


def default_class(N):
    """The untuned library default for width N (window height 16, strict
    balance, 16 waves, all N-tiles in one CTA, SPLIT24 3-term, no reorder)."""
    return class_of(1, 16, auto_ntile(N), "split24x3", 0, 16, 8)


# ----------------------------------------------------------------- features
def features(rowptr, col, m: metcf.METCF, N):
    """float32 [48] device tensor of dtc_features for CSR (device) + its METCF."""
    dev = m.RowWindowOffset.device
    rowptr = rowptr.to(dev, torch.int32).contiguous()
    col = col.to(dev, torch.int32).contiguous()
    out = torch.empty(NFEAT, dtype=torch.float32, device=dev)
    wsb = _lib.lib().dtc_features_workspace_bytes()
    ws = torch.empty(wsb, dtype=torch.uint8, device=dev)
    call("dtc_features", _ptr(rowptr), _ptr(col), m.M, col.numel(), _ptr(m.RowWindowOffset),
         _ptr(m.TCblockoffset), _ptr(m.edgeToColumn), m.nwin, m.T, N, _ptr(out), _ptr(ws),
         wsb, _stream())
    return out


# ---------------------------------------------------------------------- MLP
class MLP:
    """48 -> 64 -> 64 -> K network whose every pass runs in libdtcspmm.so."""

    def __init__(self, dims=(NFEAT, 64, 64, K), seed=0, device="cuda", params=None):
        self.dims = tuple(int(d) for d in dims)
        self.cd = MlpDims(*self.dims)
        n = _lib.lib().dtc_mlp_num_params(C.byref(self.cd))
        if n < 0:
            raise ValueError(f"bad MLP dims {dims}")
        self.n = n
        self.device = torch.device(device)
        if params is None:
            params = self.init_params(seed)
        self.params = torch.as_tensor(np.asarray(params, np.float32)).to(self.device).contiguous()
        assert self.params.numel() == n

    def init_params(self, seed):
        """He-uniform weights, zero biases (numpy, seeded)."""
        rng = np.random.default_rng(seed)
        i, h1, h2, o = self.dims
        parts = []
        for fan_in, fan_out in ((i, h1), (h1, h2), (h2, o)):
            lim = math.sqrt(6.0 / fan_in)
            parts.append(rng.uniform(-lim, lim, fan_in * fan_out))
            parts.append(np.zeros(fan_out))
        return np.concatenate(parts).astype(np.float32)

    def _acts(self, B):
        i, h1, h2, o = self.dims
        e = lambda w: torch.empty((max(B, 1), w), dtype=torch.float32, device=self.device)
        return e(h1), e(h2), e(o)

    def forward(self, X):
        X = torch.as_tensor(X, dtype=torch.float32).to(self.device).contiguous()
        B = X.shape[0]
        H1, H2, Y = self._acts(B)
        call("dtc_mlp_forward", C.byref(self.cd), _ptr(self.params), _ptr(X), B, _ptr(H1),
             _ptr(H2), _ptr(Y), _stream())
        return H1[:B], H2[:B], Y[:B]

    def loss_and_grads(self, X, target, mask):
        X = torch.as_tensor(X, dtype=torch.float32).to(self.device).contiguous()
        target = torch.as_tensor(target, dtype=torch.float32).to(self.device).contiguous()
        mask = torch.as_tensor(mask, dtype=torch.float32).to(self.device).contiguous()
        B = X.shape[0]
        H1, H2, Y = self.forward(X)
        grads = torch.empty(self.n, dtype=torch.float32, device=self.device)
        loss = torch.empty(1, dtype=torch.float32, device=self.device)
        wsb = _lib.lib().dtc_mlp_backward_workspace_bytes(C.byref(self.cd), B)
        ws = torch.empty(wsb, dtype=torch.uint8, device=self.device)
        call("dtc_mlp_backward", C.byref(self.cd), _ptr(self.params), _ptr(X), _ptr(H1),
             _ptr(H2), _ptr(Y), _ptr(target), _ptr(mask), B, _ptr(grads), _ptr(loss), _ptr(ws),
             wsb, _stream())
        return loss, grads

    def train(self, X, target, mask, steps=3000, lr=2e-3, beta1=0.9, beta2=0.999, eps=1e-8,
              batch=None, seed=0, log_every=0):
        """Adam on the masked MSE; full batch unless ``batch`` is given."""
        X = torch.as_tensor(X, dtype=torch.float32).to(self.device).contiguous()
        T = torch.as_tensor(target, dtype=torch.float32).to(self.device).contiguous()
        Mk = torch.as_tensor(mask, dtype=torch.float32).to(self.device).contiguous()
        m = torch.zeros(self.n, dtype=torch.float32, device=self.device)
        v = torch.zeros_like(m)
        rng = np.random.default_rng(seed)
        S = X.shape[0]
        hist = []
        for step in range(1, steps + 1):
            if batch and batch < S:
                idx = torch.as_tensor(rng.choice(S, batch, replace=False), device=self.device)
                xb, tb, mb = X[idx].contiguous(), T[idx].contiguous(), Mk[idx].contiguous()
            else:
                xb, tb, mb = X, T, Mk
            loss, g = self.loss_and_grads(xb, tb, mb)
            call("dtc_mlp_adam", _ptr(self.params), _ptr(g), _ptr(m), _ptr(v), self.n, lr, beta1,
                 beta2, eps, step, _stream())
            if log_every and (step % log_every == 0 or step == 1):
                hist.append((step, float(loss.item())))
        return hist

    def choose(self, X, feas):
        """Class index with the lowest predicted cost among feasible ones, per row."""
        _, _, Y = self.forward(X)
        B = Y.shape[0]
        feas = torch.as_tensor(np.asarray(feas, np.uint8)).to(self.device).contiguous()
        per_row = 1 if feas.dim() == 2 else 0
        ch = torch.empty(max(B, 1), dtype=torch.int32, device=self.device)
        call("dtc_mlp_argmin", _ptr(Y.contiguous()), _ptr(feas), per_row, B, self.dims[3],
             _ptr(ch), _stream())
        return ch[:B].cpu().numpy()

    def save(self, path, **meta):
        np.savez(path, params=self.params.cpu().numpy(), dims=np.array(self.dims), **meta)

    @classmethod
    def load(cls, path, device="cuda"):
        z = np.load(path)
        return cls(dims=tuple(z["dims"]), params=z["params"], device=device)


# -------------------------------------------------------- training targets
def targets(times):
    """times [S, K] ms (NaN = not measured) -> (log(t / t_best), mask)."""
    t = np.asarray(times, np.float64)
    ok = np.isfinite(t) & (t > 0)
    best = np.where(ok, t, np.inf).min(axis=1, keepdims=True)
    y = np.where(ok, np.log(np.where(ok, t, 1.0) / best), 0.0)
    return y.astype(np.float32), ok.astype(np.float32)


def evaluate(choices, times, N, pred=None, topk=4):
    """Regret of chosen classes vs the exhaustive best, next to the default's.
    With the model's predictions `pred` [S, K], also the regret of timing its
    `topk` cheapest predicted classes and keeping the fastest."""
    t = np.asarray(times, np.float64)
    best = np.nanmin(t, axis=1)
    pick = t[np.arange(len(t)), choices]
    dflt = np.array([t[i, default_class(int(n))] for i, n in enumerate(N)])
    reg = pick / best - 1.0
    dreg = dflt / best - 1.0
    out = dict(n=len(t), regret_mean=float(np.mean(reg)), regret_median=float(np.median(reg)),
               regret_p90=float(np.quantile(reg, 0.9)), default_regret_mean=float(np.mean(dreg)),
               speedup_vs_default_geomean=float(np.exp(np.mean(np.log(dflt / pick)))),
               exhaustive_vs_default_geomean=float(np.exp(np.mean(np.log(dflt / best)))),
               picked_reorder_frac=float(np.mean([CLASSES[c]["reorder"] for c in choices])))
    if pred is not None:
        vk = []
        for i, n in enumerate(N):
            ok = np.flatnonzero(feasible(int(n)))
            top = ok[np.argsort(np.asarray(pred[i])[ok], kind="stable")[:topk]]
            vk.append(np.nanmin(t[i, top]))
        vk = np.array(vk)
        out[f"regret_top{topk}_mean"] = float(np.mean(vk / best - 1.0))
        out[f"regret_top{topk}_median"] = float(np.median(vk / best - 1.0))
    return out


# ------------------------------------------------------- data collection
FAMILIES = ("rmat", "banded", "blockdiag", "uniform")


def sample_spec(rng, nnz_lo, nnz_hi):
    """One seeded matrix description of the training family."""
    fam = FAMILIES[int(rng.integers(len(FAMILIES)))]
    nnz = float(np.exp(rng.uniform(np.log(nnz_lo), np.log(nnz_hi))))
    spec = dict(family=fam, seed=int(rng.integers(1 << 30)), N=int(rng.choice([128, 512])),
                shuffle=int(rng.integers(2)))
    if fam == "rmat":
        a = float(rng.uniform(0.45, 0.65))
        rest = 1.0 - a
        spec.update(a=a, b=rest * 0.19 / 0.43, c=rest * 0.19 / 0.43, edge_factor=8.0,
                    scale=int(max(10, min(22, round(np.log2(nnz / 8.0 / 2.0))))))
    elif fam == "banded":
        bw = int(np.exp(rng.uniform(np.log(8), np.log(512))))
        fill = float(rng.uniform(0.1, 0.9))
        spec.update(bandwidth=bw, fill=fill, M=int(max(1024, nnz / max(1.0, 2 * bw * fill))))
    elif fam == "blockdiag":
        blk = int(np.exp(rng.uniform(np.log(32), np.log(4096))))
        deg = int(rng.integers(4, 33))
        spec.update(block=blk, degree=min(deg, blk), M=int(max(1024, nnz / min(deg, blk))))
    else:
        mean = float(np.exp(rng.uniform(np.log(4), np.log(64))))
        spec.update(mean=mean, M=int(max(1024, nnz / mean)))
    return spec


def make_matrix(spec):
    f = spec["family"]
    if f == "rmat":
        return gen.rmat(spec["scale"], spec["edge_factor"], spec["a"], spec["b"], spec["c"],
                        seed=spec["seed"])
    if f == "banded":
        return gen.banded(spec["M"], spec["bandwidth"], spec["fill"], seed=spec["seed"])
    if f == "blockdiag":
        return gen.blockdiag(spec["M"], spec["block"], spec["degree"], 0.05, seed=spec["seed"])
    return gen.uniform(spec["M"], mean=spec["mean"], seed=spec["seed"])


def measure(spec, reps=3, device="cuda"):
    """Features [48] and the measured kernel time [K] (ms; NaN = infeasible)."""
    A = make_matrix(spec)
    N = spec["N"]
    rp = torch.from_numpy(A.rowptr).to(device)
    cl = torch.from_numpy(A.col).to(device)
    vl = torch.from_numpy(A.val).to(device)
    if spec["shuffle"]:
        perm = torch.from_numpy(np.random.default_rng(spec["seed"] + 1)
                                .permutation(A.M).astype(np.int32)).to(device)
        rp, cl, vl = metcf.permute_csr(rp, cl, vl, perm)
    m = metcf.convert(rp, cl, A.M, values=vl)
    feat = features(rp, cl, m, N).cpu().numpy()
    B = torch.from_numpy(gen.normal(A.M, N, seed=spec["seed"] + 2)).to(device)
    times = np.full(K, np.nan, np.float32)
    feas = feasible(int(spec["N"])).astype(bool)
    info = dict(M=A.M, nnz=int(cl.numel()), T0=m.T)
    out = torch.empty((A.M, N), dtype=torch.float32, device=device)
    planes = {fo: metcf.pack_b(B, tune.FORMS[fo][0]) for fo in FORMS}
    for ro in (0, 1):
        src = (rp, cl, vl)
        if ro:
            t0 = time.perf_counter()
            _, rp2, c2, v2 = reorder_mod.reorder(rp, cl, vl, A.M)
            torch.cuda.synchronize()
            info["tca_s"] = time.perf_counter() - t0
            src = (rp2, c2, v2)
        for h, w in SHAPES:
            mm = m if ((h, w) == (16, 8) and not ro) else metcf.convert(src[0], src[1], A.M, H=h,
                                                                        W=w, values=src[2])
            info[f"T_r{ro}_h{h}w{w}"] = mm.T
            ws = tune.workspace_for(mm, N, B.device)
            for fo in FORMS:
                fmt, prec = tune.FORMS[fo][0], tune.FORMS[fo][1]
                scheds, _ = tune.autotune(mm, planes[fo], fmt, N, prec, reps=reps, out=out,
                                          workspace=ws)
                for s in scheds:
                    key = (s.mode, s.waves, s.ntile, fo, ro, h, w)
                    if key in _INDEX and feas[_INDEX[key]]:  # labels inside the class space
                        times[_INDEX[key]] = s.ms
            del ws, mm
    return feat, times, info


def collect(n_train, n_test, seed=0, nnz_lo=1e6, nnz_hi=3e7, reps=3, log=None, lo=0, hi=None,
            checkpoint=None, n_override=None, index_offset=0):
    """Measured dataset over seeded synthetic matrices (train, then held-out).

    The matrix list depends only on the seed and the counts, so [lo, hi) picks
    a slice that can be measured in a separate run and merged later; with
    `checkpoint` the slice measured so far is saved after every matrix. A
    matrix whose measurement fails (a workspace beyond device memory) is
    logged and left out. `n_override` fixes every matrix's N (a list drawn from
    another seed widens the training set to another width); `index_offset`
    keeps such a list's matrix indices apart from the first one's."""
    rng = np.random.default_rng(seed)
    specs = [sample_spec(rng, nnz_lo, nnz_hi) for _ in range(n_train + n_test)]
    if n_override:
        for sp in specs:
            sp["N"] = int(n_override)
    hi = len(specs) if hi is None else min(hi, len(specs))
    F, Tm, meta = [], [], []
    for i in range(lo, hi):
        sp = specs[i]
        t0 = time.perf_counter()
        try:
            f, t, info = measure(sp, reps=reps)
        except (torch.OutOfMemoryError, RuntimeError) as e:  # e.g. a workspace above device memory
            torch.cuda.empty_cache()
            if log:
                log(f"[{i + 1}/{len(specs)}] {sp['family']} skipped: {str(e).splitlines()[0][:160]}")
            continue
        F.append(f)
        Tm.append(t)
        meta.append(dict(sp, **info, index=i + index_offset,
                         split="train" if i < n_train else "test"))
        if log:
            log(f"[{i + 1}/{len(specs)}] {sp['family']} N={sp['N']} nnz={info['nnz']} "
                f"best={np.nanmin(t):.3f}ms {time.perf_counter() - t0:.1f}s")
        if checkpoint:
            save_dataset(dict(features=np.stack(F), times=np.stack(Tm), meta=meta), checkpoint)
    return dict(features=np.stack(F), times=np.stack(Tm), meta=meta)


def merge(parts):
    """One dataset from slices measured separately (ordered by matrix index);
    times of classes infeasible for a matrix's N are set to NaN."""
    F = np.concatenate([p["features"] for p in parts])
    Tm = np.concatenate([p["times"] for p in parts]).astype(np.float64)
    meta = sum((p["meta"] for p in parts), [])
    for i, m in enumerate(meta):
        Tm[i, ~feasible(int(m["N"])).astype(bool)] = np.nan
    order = np.argsort([m["index"] for m in meta], kind="stable")
    return dict(features=F[order], times=Tm[order], meta=[meta[i] for i in order])


def save_dataset(ds, path=DATASET_PATH):
    import json
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.savez_compressed(path, features=ds["features"], times=ds["times"],
                        meta=np.array(json.dumps(ds["meta"])))


def load_dataset(path=DATASET_PATH):
    import json
    z = np.load(path)
    return dict(features=z["features"], times=z["times"], meta=json.loads(str(z["meta"])))


def split(ds):
    tr = np.array([m["split"] == "train" for m in ds["meta"]])
    N = np.array([m["N"] for m in ds["meta"]])
    return tr, N


def fit(ds, steps=3000, lr=2e-3, seed=0, device="cuda"):
    """Trains on the dataset's train split; returns (model, held-out evaluation)."""
    tr, N = split(ds)
    y, mk = targets(ds["times"])
    net = MLP(seed=seed, device=device)
    net.train(ds["features"][tr], y[tr], mk[tr], steps=steps, lr=lr, seed=seed)
    feas = np.stack([feasible(int(n)) for n in N[~tr]])
    ch = net.choose(ds["features"][~tr], feas)
    _, _, Y = net.forward(ds["features"][~tr])
    return net, evaluate(ch, ds["times"][~tr], N[~tr], pred=Y.cpu().numpy())


# ------------------------------------------------------------- scheduler
@dataclass
class Plan:
    cls: int
    H: int
    W: int
    form: str
    reorder: bool
    mode: int
    waves: int
    ntile: int
    source: str  # "model" or "exhaustive"


class Scheduler:
    """Picks a class for (matrix, N): the trained model when its weights are
    present and match the class space, else the exhaustive autotuner over every
    class."""

    def __init__(self, weights=WEIGHTS_PATH, device="cuda"):
        self.net = MLP.load(weights, device) if weights and os.path.exists(weights) else None
        if self.net is not None and self.net.dims != (NFEAT, 64, 64, K):
            self.net = None  # weights of another class space: fall back

    def plan(self, rowptr, col, m: metcf.METCF, N, exhaustive=False, B=None, reps=3,
             verify_top=0):
        """The class to run. With verify_top = k > 1 the model's k cheapest
        predicted classes are timed on the caller's data and the fastest wins
        (model-guided search: k measurements instead of all K classes)."""
        if self.net is not None and not exhaustive:
            f = features(rowptr, col, m, N).reshape(1, -1)
            if verify_top > 1:
                _, _, Y = self.net.forward(f)
                y = Y[0].cpu().numpy()
                ok = np.flatnonzero(feasible(N))
                top = ok[np.argsort(y[ok], kind="stable")[:verify_top]]
                c = self._fastest(rowptr, col, m, N, B, reps, [int(i) for i in top])
                src = "model+verify"
            else:
                c = int(self.net.choose(f, feasible(N))[0])
                src = "model"
        else:
            c = self._exhaustive(rowptr, col, m, N, B, reps)
            src = "exhaustive"
        k = CLASSES[c]
        return Plan(c, k["H"], k["W"], k["form"], bool(k["reorder"]), k["mode"], k["waves"],
                    k["ntile"], src)

    @staticmethod
    def _fastest(rowptr, col, m, N, B, reps, classes):
        """Times the given classes on this matrix (CUDA events) and returns the fastest."""
        dev = m.RowWindowOffset.device
        if B is None:
            B = torch.randn((m.M, N), device=dev)
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        mets, perms, best, best_c = {}, {}, None, None
        out = torch.empty((m.M, N), dtype=torch.float32, device=dev)
        for c in classes:
            k = CLASSES[c]
            key = (k["reorder"], k["H"], k["W"])
            if key not in mets:
                if k["reorder"]:
                    if "p" not in perms:
                        perms["p"] = reorder_mod.reorder(rowptr.to(dev), col.to(dev), None, m.M)
                    _, rp2, c2, _ = perms["p"]
                    mets[key] = metcf.convert(rp2, c2, m.M, H=k["H"], W=k["W"])
                else:
                    mets[key] = m if (k["H"], k["W"]) == (m.H, m.W) else metcf.convert(
                        rowptr.to(dev), col.to(dev), m.M, H=k["H"], W=k["W"])
            mm = mets[key]
            fmt, prec = tune.FORMS[k["form"]][0], tune.FORMS[k["form"]][1]
            planes = metcf.pack_b(B, fmt)
            sched = tune.Schedule(mode=k["mode"], waves=k["waves"], ntile=k["ntile"],
                                  grid=min(k["waves"] * sms, max(mm.T, 1)), ms=0.0)
            ws = tune.workspace_for(mm, N, dev)
            tune.run(mm, planes, fmt, N, prec, sched, out=out, workspace=ws)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                tune.run(mm, planes, fmt, N, prec, sched, out=out, workspace=ws)
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            if best is None or ms < best:
                best, best_c = ms, c
        return best_c

    @staticmethod
    def _exhaustive(rowptr, col, m, N, B, reps):
        dev = m.RowWindowOffset.device
        if B is None:
            B = torch.randn((m.M, N), device=dev)
        best, best_c = None, None
        for ro in (0, 1):
            src = (rowptr.to(dev), col.to(dev), m.TCvalues)
            if ro:
                _, rp2, c2, _ = reorder_mod.reorder(src[0], src[1], None, m.M)
                src = (rp2, c2, None)
            for h, w in SHAPES:
                mm = m if ((h, w) == (m.H, m.W) and not ro) else metcf.convert(
                    src[0], src[1], m.M, H=h, W=w)
                for fo in FORMS:
                    fmt, prec = tune.FORMS[fo][0], tune.FORMS[fo][1]
                    scheds, b = tune.autotune(mm, metcf.pack_b(B, fmt), fmt, N, prec, reps=reps)
                    ok = feasible(N)
                    for sc in scheds:  # the fastest schedule inside the class space
                        key = (sc.mode, sc.waves, sc.ntile, fo, ro, h, w)
                        if key in _INDEX and ok[_INDEX[key]] and (best is None or sc.ms < best):
                            best, best_c = sc.ms, _INDEX[key]
        return best_c


def main(argv=None):
    """python -m dtc_b200.costmodel collect|merge|train ... (dataset + weights under data/)."""
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["collect", "merge", "train"])
    ap.add_argument("--range", default=None, help="lo:hi slice of the matrix list (collect)")
    ap.add_argument("--out", default=None, help="slice file (collect --range)")
    ap.add_argument("--parts", nargs="*", default=[], help="slice files (merge)")
    ap.add_argument("--N", type=int, default=0, help="fixed N for every matrix (collect)")
    ap.add_argument("--index-offset", type=int, default=0, help="added to matrix indices")
    ap.add_argument("--train", type=int, default=400)
    ap.add_argument("--test", type=int, default=100)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--nnz-lo", type=float, default=1e6)
    ap.add_argument("--nnz-hi", type=float, default=3e7)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--dataset", default=DATASET_PATH)
    ap.add_argument("--weights", default=WEIGHTS_PATH)
    a = ap.parse_args(argv)
    if a.cmd == "collect" and a.range:
        lo, hi = (int(x) for x in a.range.split(":"))
        collect(a.train, a.test, a.seed, a.nnz_lo, a.nnz_hi, a.reps, log=print, lo=lo, hi=hi,
                checkpoint=a.out, n_override=a.N or None, index_offset=a.index_offset)
        return
    if a.cmd == "collect":
        ds = collect(a.train, a.test, a.seed, a.nnz_lo, a.nnz_hi, a.reps, log=print)
        save_dataset(ds, a.dataset)
    if a.cmd == "merge":
        save_dataset(merge([load_dataset(p) for p in a.parts]), a.dataset)
    ds = load_dataset(a.dataset)
    net, ev = fit(ds, steps=a.steps, seed=a.seed)
    net.save(a.weights, eval=np.array(str(ev)))
    print(ev)


if __name__ == "__main__":
    main()
