"""ORACLE -- test infrastructure only (the checker, never the product path).

FP64 numpy restatements of the learned cost model's pieces, to check the
library's CUDA kernels:
* ``features``: the 48-dimensional structural feature vector (dtc_features),
  from CSR and the oracle's ME-TCF arrays;
* ``forward`` / ``backward``: the MLP in -> h1 -> h2 -> out with ReLU hidden
  layers and the masked-MSE loss, by the chain rule written out by hand;
* ``adam``: one bias-corrected Adam step.
Parameter layout: W1[h1][in], b1[h1], W2[h2][h1], b2[h2], W3[out][h2], b3[out].
"""
import numpy as np


def _log_bin(v, nbins):
    v = np.asarray(v, np.int64)
    b = np.floor(np.log2(np.maximum(v, 1))).astype(np.int64) + 1
    return np.minimum(b, nbins - 1)


def features(rowptr, col, M, m, N):
    """m: dict from oracle.metcf (RowWindowOffset, TCblockoffset, edgeToColumn, T)."""
    rowptr = np.asarray(rowptr, np.int64)
    col = np.asarray(col, np.int64)
    nnz = int(rowptr[-1])
    nwin = (M + 15) // 16
    T = int(m["T"])
    f = np.zeros(48, np.float64)
    lens = np.diff(rowptr)
    rb = np.where(lens == 0, 0, _log_bin(lens, 16))
    f[0:16] = np.bincount(rb, minlength=16)[:16] / max(M, 1)
    rwo = np.asarray(m["RowWindowOffset"], np.int64)
    bp = np.diff(rwo)
    wb = np.where(bp == 0, 0, _log_bin(bp, 12))
    f[16:28] = np.bincount(wb, minlength=12)[:12] / max(nwin, 1)
    toff = np.asarray(m["TCblockoffset"], np.int64)
    nb = np.diff(toff)
    bb = np.minimum(np.where(nb <= 1, 0, np.floor(np.log2(np.maximum(nb, 1))).astype(np.int64)), 7)
    f[28:36] = np.bincount(bb, minlength=8)[:8] / max(T, 1)
    e2c = np.asarray(m["edgeToColumn"], np.int64)
    U = 0
    for w in range(nwin):
        e0, e1 = rowptr[w * 16], rowptr[min(w * 16 + 16, M)]
        U += int(e2c[e0:e1].max()) + 1 if e1 > e0 else 0
    rows = np.repeat(np.arange(M), lens)
    dist = np.abs(col - rows)
    mm, w_, t_, z = max(M, 1), max(nwin, 1), max(T, 1), max(nnz, 1)
    f[36] = np.log2(mm) / 24.0
    f[37] = np.log2(z) / 28.0
    f[38] = np.log2(t_) / 26.0
    f[39] = np.log2(max(N, 1)) / 10.0
    f[40] = np.log2(z / mm) / 10.0
    f[41] = np.log2(max(int(lens.max()) if M else 1, 1)) / 16.0
    f[42] = U / z
    f[43] = 8.0 * T / U if U > 0 else 1.0
    f[44] = int(dist.sum()) / z / mm
    f[45] = int((dist < 64).sum()) / z
    mean = T / w_
    var = int((bp * bp).sum()) / w_ - mean * mean
    f[46] = np.sqrt(max(var, 0.0)) / mean / 10.0 if mean > 0 else 0.0
    f[47] = np.count_nonzero(bp == 0) / w_
    return f.astype(np.float32)


def unpack(params, dims):
    i, h1, h2, o = dims
    p = np.asarray(params, np.float64)
    k = 0
    out = []
    for shape in ((h1, i), (h1,), (h2, h1), (h2,), (o, h2), (o,)):
        n = int(np.prod(shape))
        out.append(p[k:k + n].reshape(shape))
        k += n
    assert k == len(p)
    return out


def forward(params, dims, X):
    W1, b1, W2, b2, W3, b3 = unpack(params, dims)
    X = np.asarray(X, np.float64)
    H1 = np.maximum(X @ W1.T + b1, 0.0)
    H2 = np.maximum(H1 @ W2.T + b2, 0.0)
    Y = H2 @ W3.T + b3
    return H1, H2, Y


def loss_and_grads(params, dims, X, target, mask):
    W1, b1, W2, b2, W3, b3 = unpack(params, dims)
    X = np.asarray(X, np.float64)
    H1, H2, Y = forward(params, dims, X)
    mk = np.asarray(mask, np.float64)
    msum = mk.sum() if mk.sum() > 0 else 1.0
    D = Y - np.asarray(target, np.float64)
    loss = (mk * D * D).sum() / msum
    dY = 2.0 * mk * D / msum
    gW3, gb3 = dY.T @ H2, dY.sum(0)
    dH2 = (dY @ W3) * (H2 > 0)
    gW2, gb2 = dH2.T @ H1, dH2.sum(0)
    dH1 = (dH2 @ W2) * (H1 > 0)
    gW1, gb1 = dH1.T @ X, dH1.sum(0)
    g = np.concatenate([a.ravel() for a in (gW1, gb1, gW2, gb2, gW3, gb3)])
    return loss, g


def adam(p, g, m, v, lr, b1, b2, eps, step):
    p, g, m, v = (np.asarray(a, np.float64) for a in (p, g, m, v))
    m = b1 * m + (1 - b1) * g
    v = b2 * v + (1 - b2) * g * g
    c1, c2 = 1 - b1 ** step, 1 - b2 ** step
    return p - lr * (m / c1) / (np.sqrt(v / c2) + eps), m, v
