"""Deterministic small CSR cases shared by the golden-vector generator and the tests.

Each case returns (rowptr int32[M+1], col int32[nnz], val float32[nnz], M).
They cover the edge cases the conversion and the SpMM must get right:
M % 16 != 0, empty rows, empty windows, duplicate (row, col) pairs, windows
with > 255 distinct columns, a hub row, unsorted columns inside rows.
"""
import numpy as np


def _from_rows(rows, M):
    rowptr = np.zeros(M + 1, np.int32)
    rowptr[1:] = np.cumsum([len(r) for r in rows])
    col = np.concatenate([np.asarray(r, np.int32) for r in rows]) if rowptr[-1] else \
        np.zeros(0, np.int32)
    return rowptr, col.astype(np.int32)


def _vals(n, seed):
    return np.random.default_rng(seed).uniform(-1, 1, n).astype(np.float32)


def small_uniform(seed=1):
    rng = np.random.default_rng(seed)
    M = 100
    rows = [np.sort(rng.choice(M, size=min(M, rng.poisson(5)), replace=False)) for _ in range(M)]
    rows = [r if len(r) else np.array([i % M]) for i, r in enumerate(rows)]  # no empty windows
    rp, c = _from_rows(rows, M)
    return rp, c, _vals(len(c), seed + 100), M


def uniform_4096(seed=0):
    """The small benchmark shape: 4096 x 4096, Poisson(8) rows (numpy-generated)."""
    rng = np.random.default_rng(seed)
    M = 4096
    rows = [np.sort(rng.choice(M, size=rng.poisson(8), replace=False)) for _ in range(M)]
    rp, c = _from_rows(rows, M)
    return rp, c, _vals(len(c), seed + 100), M


def empty_windows(seed=2):
    """Rows 16..47 empty (windows 1 and 2 have no TC blocks), other scattered empty rows."""
    rng = np.random.default_rng(seed)
    M = 83
    rows = []
    for i in range(M):
        if 16 <= i < 48 or i % 7 == 3:
            rows.append([])
        else:
            rows.append(np.sort(rng.choice(M, size=rng.integers(1, 6), replace=False)))
    rp, c = _from_rows(rows, M)
    return rp, c, _vals(len(c), seed + 100), M


def duplicates(seed=3):
    rng = np.random.default_rng(seed)
    M = 40
    rows = []
    for i in range(M):
        base = rng.choice(M, size=rng.integers(1, 6), replace=False)
        dup = rng.choice(base, size=rng.integers(0, 3))       # repeated columns
        r = np.concatenate([base, dup])
        rng.shuffle(r)                                         # unsorted inside the row
        rows.append(r)
    rp, c = _from_rows(rows, M)
    return rp, c, _vals(len(c), seed + 100), M


def wide_window(seed=4):
    """Window 0 touches 600 distinct columns (75 TC blocks, > 255 distinct ids)."""
    rng = np.random.default_rng(seed)
    M = 1000
    rows = []
    for i in range(M):
        k = 60 if i < 16 else int(rng.integers(1, 4))
        rows.append(np.sort(rng.choice(M, size=k, replace=False)))
    rp, c = _from_rows(rows, M)
    return rp, c, _vals(len(c), seed + 100), M


def hub(seed=5):
    """One row with 3000 entries in an otherwise sparse 4000 x 4000 matrix; M % 16 == 0."""
    rng = np.random.default_rng(seed)
    M = 4000
    rows = []
    for i in range(M):
        k = 3000 if i == 37 else int(rng.integers(1, 5))
        rows.append(np.sort(rng.choice(M, size=k, replace=False)))
    rp, c = _from_rows(rows, M)
    return rp, c, _vals(len(c), seed + 100), M


def rmat12(seed=7):
    """R-MAT (0.57, 0.19, 0.19, 0.05), 2^12 nodes, 16 * 2^12 generated edges,
    symmetrised, self-loops added, duplicates removed (numpy-generated): the
    power-law shape of the benchmark at a size the golden files can carry."""
    rng = np.random.default_rng(seed)
    scale, M = 12, 1 << 12
    ne = 16 * M
    probs = np.array([0.57, 0.19, 0.19, 0.05])
    src = np.zeros(ne, np.int64)
    dst = np.zeros(ne, np.int64)
    for _ in range(scale):
        q = rng.choice(4, size=ne, p=probs)
        src = 2 * src + (q >> 1)
        dst = 2 * dst + (q & 1)
    r = np.concatenate([src, dst, np.arange(M)])
    c = np.concatenate([dst, src, np.arange(M)])
    key = np.unique(r * M + c)
    r, c = key // M, key % M
    rowptr = np.zeros(M + 1, np.int32)
    rowptr[1:] = np.cumsum(np.bincount(r, minlength=M))
    col = c.astype(np.int32)
    return rowptr, col, _vals(len(col), seed + 100), M


def banded_dense(seed=6):
    """Dense band: full 16 x 8 TC blocks (128 nonzeros per block)."""
    M = 256
    rows = [np.arange(max(0, i - 20), min(M, i + 21)) for i in range(M)]
    rp, c = _from_rows(rows, M)
    return rp, c, _vals(len(c), seed + 100), M


CASES = {
    "small_uniform": small_uniform,
    "uniform_4096": uniform_4096,
    "empty_windows": empty_windows,
    "duplicates": duplicates,
    "wide_window": wide_window,
    "hub": hub,
    "banded_dense": banded_dense,
    "rmat12": rmat12,
}

# cases the reference's CPU `preprocess` handles safely (it has no empty-window
# guard: DTC-SpMM/DTCSpMM.cpp:281-297)
CPU_REFERENCE_SAFE = ["small_uniform", "uniform_4096", "duplicates", "wide_window", "hub",
                      "banded_dense", "rmat12"]

# (block_h, block_w) shapes the reference's preprocess_gpu was run with. The
# 16 x 8 files keep their original names (ref_gpu_<case>.npz); the others carry
# the shape: ref_gpu_h<H>w<W>__<case>.npz.
GOLDEN_SHAPES = [(16, 8), (32, 8), (16, 16)]


def golden_name(case, H=16, W=8):
    return f"ref_gpu_{case}.npz" if (H, W) == (16, 8) else f"ref_gpu_h{H}w{W}__{case}.npz"


def parse_golden_name(fname):
    """ref_gpu_[h<H>w<W>__]<case>.npz -> (case, H, W)."""
    stem = fname[len("ref_gpu_"):-len(".npz")]
    if "__" in stem:
        shape, case = stem.split("__", 1)
        H, W = shape[1:].split("w")
        return case, int(H), int(W)
    return stem, 16, 8
