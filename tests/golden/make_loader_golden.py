"""Generates tests/golden/ref_loader_<case>.npz from the reference's own graph
loader, scripts/DTCSpMM/dataset.py (DTC_dataset, run unmodified: it needs
only torch, numpy and scipy).

Each case is a synthetic src_li / dst_li / num_nodes file in the format the
loader reads (duplicate edges, self-loops, unsorted edges, isolated nodes
including the last one). The fixture stores the inputs and the loader's
row_pointers and column_index.

Run in a container that holds the reference sources (DTC_REFERENCE_ROOT,
default /root/reference): python tests/golden/make_loader_golden.py
"""
import importlib.util
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_ROOT = os.environ.get("DTC_REFERENCE_ROOT", "/root/reference")
LOADER = os.path.join(REF_ROOT, "scripts", "DTCSpMM", "dataset.py")


def edges(seed, n, m, dup, isolated):
    rng = np.random.default_rng(seed)
    live = np.setdiff1d(np.arange(n), rng.choice(n - 1, isolated, replace=False))
    live = live[live != n - 1]                      # the last node has no edges
    s = rng.choice(live, m).astype(np.int64)
    d = rng.choice(live, m).astype(np.int64)
    s[:dup], d[:dup] = s[m - dup:], d[m - dup:]     # duplicate edges
    s[dup:dup + 16] = d[dup:dup + 16]               # self-loops
    return s, d, n


CASES = {
    "small": (0, 64, 400, 30, 5),
    "medium": (1, 2000, 12000, 800, 80),
    "dense_dups": (2, 200, 20000, 9000, 3),
}


def _reference_loader():
    spec = importlib.util.spec_from_file_location("ref_dtc_dataset", LOADER)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.DTC_dataset


def main():
    DTC_dataset = _reference_loader()
    with tempfile.TemporaryDirectory() as d:
        for name, args in CASES.items():
            s, t, n = edges(*args)
            path = os.path.join(d, name + ".npz")
            np.savez(path, src_li=s, dst_li=t, num_nodes=np.int64(n))
            g = DTC_dataset(path)
            rp = g.row_pointers.numpy().astype(np.int32)
            col = g.column_index.numpy().astype(np.int32)
            np.savez_compressed(os.path.join(HERE, f"ref_loader_{name}.npz"), src_li=s, dst_li=t,
                                num_nodes=np.int64(n), row_pointers=rp, column_index=col)
            print(f"{name}: {n} nodes, {len(s)} edges -> {int(rp[-1])} CSR entries")


if __name__ == "__main__":
    main()
