"""Generates tests/golden/ref_tca_<case>.npz: the reference's own TCA reorder
(reordering/TCA_reorder.py, run unmodified) on small symmetric graphs.

The script imports datasketch, libMHCUDA, cuGraph and cudf, none of which are
installed. It runs here with small stand-in modules that supply its inputs
and nothing else, so its merge queue, union-find, cluster caps, requeue rule,
level-2 clustering and output order (TCA_reorder.py:83-315) are the
reference's own code:

* MinHash / MinHashLSH (both levels): the "signature" of a row or cluster is
  its exact column set, and a query returns, in insertion order, every key
  whose set has exact Jaccard >= the index's threshold (0.2 at both levels in
  the script) -- the exact rule MinHash LSH approximates. Keys come back as
  ints: with numpy 2 the script's np.concatenate of the float pair buffer
  with an array of datasketch's string keys fails.
* cugraph.jaccard: the exact Jaccard of the two vertices' neighbourhoods in
  the undirected graph (the union of both edge directions); the graphs here
  are symmetric, so that is the Jaccard of the two CSR rows, the value the
  script's own jd() gives for requeued pairs.
* The dataset load and the two result files go to memory (np.load / np.savez
  are redirected for the script's run); nothing is written anywhere else.

Each fixture also holds the reference pipeline's reordered CSR: the script's
relabelled edge list (its second result file) read by the reference's own
graph loader (scripts/DTCSpMM/dataset.py, see make_loader_golden.py).

The one detail the script leaves open is the order of equal similarities:
its Pair.__lt__ compares similarity alone, so Python's heap pops tied pairs
in an order fixed by the heap's history (and, through the insertion order, by
cuGraph's output order). The library fixes it: among the pairs of the highest
similarity, the smallest (p1, p2) first. The script's queue is replaced, for
its run, by a PriorityQueue subclass that pops that pair and otherwise works
as before; every other step runs as written. Ties are common (most pops on
these graphs meet one), and each fixture records how many pops of each level
met a tie.

Graphs: stochastic block models with self-loops (no empty rows: the script
skips an empty row before its every-1000-rows flush check,
TCA_reorder.py:121-126, so an empty last row would drop the candidates
gathered since the last flush; the library does not reproduce that).

Run in a container that holds the reference sources (DTC_REFERENCE_ROOT,
default /root/reference): python tests/golden/make_tca_golden.py
"""
import contextlib
import heapq
import io
import os
import queue
import runpy
import sys
import tempfile
import types

import numpy as np

import make_loader_golden  # this folder: the reference graph loader

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("DTC_REFERENCE_ROOT", "/root/reference")
SCRIPT = os.path.join(REF_ROOT, "reordering", "TCA_reorder.py")

# name: (seed, nodes, block sizes range, p_in, p_out, --thres)
CASES = {
    "sbm240_t4": (1, 240, (4, 14), 0.55, 0.01, 4),
    "sbm320_t8": (2, 320, (6, 20), 0.5, 0.008, 8),
    "sbm400_t16": (3, 400, (8, 28), 0.45, 0.006, 16),
    "sbm300_t2": (4, 300, (3, 9), 0.7, 0.012, 2),
    # two graphs on which the orientation of a requeued pair (root(p1),
    # root(p2)) changes the result: it decides which root an equal-size merge
    # keeps, and later requeues use that root row's own column set
    "sbm200_t8": (5, 200, (3, 7), 0.5, 0.008, 8),
    "sbm240_t6": (5, 240, (3, 12), 0.45, 0.01, 6),
}


def sbm(seed, n, sizes, p_in, p_out):
    """Symmetric stochastic-block graph with self-loops, node ids shuffled."""
    rng = np.random.default_rng(seed)
    blocks, left = [], n
    while left > 0:
        b = min(left, int(rng.integers(sizes[0], sizes[1] + 1)))
        blocks.append(b)
        left -= b
    label = np.repeat(np.arange(len(blocks)), blocks)
    same = label[:, None] == label[None, :]
    prob = np.where(same, p_in, p_out)
    upper = np.triu(rng.random((n, n)) < prob, 1)
    adj = upper | upper.T | np.eye(n, dtype=bool)
    perm = rng.permutation(n)
    adj = adj[np.ix_(perm, perm)]
    src, dst = np.nonzero(adj)
    return src.astype(np.int64), dst.astype(np.int64), n


def _jac(a, b):
    if not a or not b:
        return 0.0
    inter = len(a & b)
    return inter / len(a | b)


def _stub_modules():
    class MinHash:
        def __init__(self, num_perm=128, **kw):
            self.items = set()

        def update(self, b):
            self.items.add(b)

    class WeightedMinHash:
        def __init__(self, seed, hashvalues):
            self.items = hashvalues

    class WeightedMinHashGenerator:
        def __init__(self, dim, *a, **kw):
            self.rs = self.ln_cs = self.betas = None

    class MinHashLSH:
        def __init__(self, threshold=0.9, num_perm=128, **kw):
            self.threshold, self.keys, self.sets = threshold, [], []

        def insert(self, key, m):
            self.keys.append(int(key))
            self.sets.append(m.items)

        def query(self, m):
            return [k for k, s in zip(self.keys, self.sets) if _jac(m.items, s) >= self.threshold]

    ds = types.ModuleType("datasketch")
    ds.MinHash, ds.MinHashLSH = MinHash, MinHashLSH
    ds.WeightedMinHash, ds.WeightedMinHashGenerator = WeightedMinHash, WeightedMinHashGenerator

    mh = types.ModuleType("libMHCUDA")
    mh.minhash_cuda_init = lambda *a, **kw: object()
    mh.minhash_cuda_assign_vars = lambda *a, **kw: None
    mh.minhash_cuda_fini = lambda *a, **kw: None

    def calc(gen, csr):
        ptr, idx = np.asarray(csr.indptr), np.asarray(csr.indices)
        return [frozenset(int(x) for x in idx[ptr[i]:ptr[i + 1]]) for i in range(len(ptr) - 1)]
    mh.minhash_cuda_calc = calc

    cudf = types.ModuleType("cudf")

    class DataFrame(dict):
        pass
    cudf.DataFrame = DataFrame
    cudf.Series = lambda x: np.asarray(x)

    cg = types.ModuleType("cugraph")

    class Graph:
        def from_cudf_edgelist(self, df, source, destination, edge_attr=None):
            nb = {}
            for s, d in zip(np.asarray(df[source]).tolist(), np.asarray(df[destination]).tolist()):
                nb.setdefault(int(s), set()).add(int(d))
                nb.setdefault(int(d), set()).add(int(s))
            self.nb = nb
    cg.Graph = Graph

    class _Result:
        def __init__(self, rows):
            self.values = np.array(rows, np.float64).reshape(-1, 3)

        def to_pandas(self):
            return self

    def jaccard(G, pairs):
        rows = []
        for a, b in zip(np.asarray(pairs["first"]).tolist(), np.asarray(pairs["second"]).tolist()):
            a, b = int(a), int(b)
            rows.append((_jac(G.nb.get(a, set()), G.nb.get(b, set())), a, b))
        return _Result(rows)
    cg.jaccard = jaccard
    return {"datasketch": ds, "libMHCUDA": mh, "cudf": cudf, "cugraph": cg}


class TieOrderedQueue(queue.PriorityQueue):
    """The script's priority queue with ties broken by (p1, p2) ascending.

    Pops, among the queued Pairs of the highest similarity, the one with the
    smallest (p1, p2); counts pops and the pops that met a tie."""
    made = []

    def _init(self, maxsize):
        super()._init(maxsize)
        self.pops = self.ties = 0
        TieOrderedQueue.made.append(self)

    def _get(self):
        top = self.queue[0].simi
        tied = [i for i, x in enumerate(self.queue) if x.simi == top]
        self.pops += 1
        if len(tied) == 1:
            return super()._get()
        self.ties += 1
        k = min(tied, key=lambda i: (self.queue[i].p1, self.queue[i].p2))
        item = self.queue[k]
        self.queue[k] = self.queue[-1]
        self.queue.pop()
        heapq.heapify(self.queue)
        return item


def run_reference(src, dst, n, thres, name="case"):
    """The reference script on (src, dst, n) -> (reorder_id, per-level stats)."""
    store = {}
    stubs = _stub_modules()
    saved_mods = {k: sys.modules.get(k) for k in stubs}
    saved = (np.load, np.savez, queue.PriorityQueue, list(sys.argv))

    def fake_load(path, *a, **kw):
        assert str(path).endswith(name + ".npz"), path
        return {"src_li": src, "dst_li": dst, "num_nodes": np.int64(n)}

    def fake_savez(path, **kw):
        store[os.path.basename(str(path))] = kw

    TieOrderedQueue.made = []
    try:
        sys.modules.update(stubs)
        np.load, np.savez, queue.PriorityQueue = fake_load, fake_savez, TieOrderedQueue
        sys.argv = ["TCA_reorder.py", "--dataset", name, "--thres", str(thres)]
        with contextlib.redirect_stdout(io.StringIO()):
            runpy.run_path(SCRIPT, run_name="__main__")
    finally:
        np.load, np.savez, queue.PriorityQueue, sys.argv[:] = saved[0], saved[1], saved[2], saved[3]
        for k, v in saved_mods.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
    reorder = np.asarray(store[name + ".reorder_id.npz"]["reorder_id"], np.int32)
    stats = [(q.pops, q.ties) for q in TieOrderedQueue.made]
    run_reference.relabelled = store[name + ".reorder.npz"]
    return reorder, stats


def main():
    if not os.path.exists(SCRIPT):
        raise SystemExit(f"reference script not found: {SCRIPT}")
    for name, (seed, n, sizes, p_in, p_out, thres) in CASES.items():
        src, dst, n = sbm(seed, n, sizes, p_in, p_out)
        reorder, stats = run_reference(src, dst, n, thres, name)
        assert len(stats) == 2, stats
        print(f"{name}: pops {[p for p, _ in stats]}, pops that met a tie {[t for _, t in stats]}")
        # the reference pipeline's reordered CSR: the script's relabelled edge
        # list (TCA_reorder.py:316-326) read back by its graph loader
        rel = run_reference.relabelled
        with tempfile.TemporaryDirectory() as d:
            path = os.path.join(d, name + ".reorder.npz")
            np.savez(path, src_li=np.asarray(rel["src_li"], np.int64),
                     dst_li=np.asarray(rel["dst_li"], np.int64), num_nodes=np.int64(n))
            g = make_loader_golden._reference_loader()(path)
            rrp = g.row_pointers.numpy().astype(np.int32)
            rcol = g.column_index.numpy().astype(np.int32)
        np.savez_compressed(os.path.join(HERE, f"ref_tca_{name}.npz"), src_li=src, dst_li=dst,
                            num_nodes=np.int64(n), thres=np.int64(thres), reorder_id=reorder,
                            reordered_row_pointers=rrp, reordered_column_index=rcol,
                            pops=np.array([p for p, _ in stats], np.int64),
                            ties=np.array([t for _, t in stats], np.int64))


if __name__ == "__main__":
    main()
