"""ORACLE -- test infrastructure only (the checker, never the product path).

CPU restatement of the TCA reorder (reordering/TCA_reorder.py:53-326) with the
hash functions, LSH banding and candidate-pair rule of the library's
dtc_tca_reorder, so that the library's permutation can be checked bit-exactly:

* MinHash: h_k(c) = high 32 bits of mix64(c ^ salt_k), salt_k =
  mix64(seed + 0x9e3779b97f4a7c15 * (k + 1)), mix64 = the splitmix64
  finaliser; signature = min over the item's set (0xffffffff when empty).
* LSH: band b hashes its rows_per_band values v_j as h = mix64(h ^ v_j) from
  h = 0x51ed27a3c0ffee11 ^ b; key = b << 40 | (h mod 2^40); empty items are
  left out. Keys are sorted stably (items ascending within a bucket) and each
  position pairs with the next bucket_window positions of the same key.
* Greedy merge (TCA_reorder.py:171-205, :268-293): pop pairs by descending
  Jaccard, ties by (lo, hi) ascending; merge two live roots (smaller into
  larger, equal sizes into the first); a cluster reaching the cap is closed;
  a pair whose ends are not both roots is requeued once as (root, root) with
  the Jaccard of the roots' own sets.
* Output order (TCA_reorder.py:308-315): level-2 groups by first appearance,
  their clusters ascending, each cluster's rows ascending.

The reference's own MinHash and LSH come from datasketch / libMHCUDA and its
Jaccard from cuGraph, none of which are installed, so the library's LSH
candidates are not comparable to the reference's. Everything after the
candidates (two_level: the merge, level 2 and the output order) is pinned to
the reference script itself: tests/golden/ref_tca_*.npz hold its reorder_id
for candidates given by threshold_pairs (tests/golden/make_tca_golden.py).
The one open detail, the order of equal similarities (the script's Pair
compares similarity only), is (p1, p2) ascending here and in those fixtures.
"""
import heapq

import numpy as np

M64 = (1 << 64) - 1
GOLD = 0x9E3779B97F4A7C15


def _mix64_np(z):
    z = np.asarray(z, np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _mix64(z):
    z &= M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
    return z ^ (z >> 31)


DEFAULTS = dict(num_perm=128, bands=42, rows_per_band=3, thres=16, c_thres=128,
                bucket_window=8, seed=2022)


def signatures(sets, P, seed):
    """sets: list of sorted int arrays -> uint32 [n, P]."""
    salts = np.array([_mix64(seed + GOLD * (k + 1)) for k in range(P)], np.uint64)
    sig = np.full((len(sets), P), 0xFFFFFFFF, np.uint64)
    for i, s in enumerate(sets):
        if len(s):
            h = _mix64_np(np.asarray(s, np.uint64)[:, None] ^ salts[None, :]) >> np.uint64(32)
            sig[i] = h.min(axis=0)
    return sig.astype(np.uint32)


def lsh_pairs(sig, bands, rpb, win):
    n = sig.shape[0]
    keys, items = [], []
    for b in range(bands):
        for i in range(n):
            vals = [int(v) for v in sig[i, b * rpb:(b + 1) * rpb]]
            if any(v == 0xFFFFFFFF for v in vals):
                keys.append(M64)
            else:
                h = 0x51ED27A3C0FFEE11 ^ b
                for v in vals:
                    h = _mix64(h ^ v)
                keys.append((b << 40) | (h & ((1 << 40) - 1)))
            items.append(i)
    order = sorted(range(len(keys)), key=lambda t: (keys[t], t))  # stable
    ks = [keys[t] for t in order]
    it = [items[t] for t in order]
    pairs = set()
    for p in range(len(ks)):
        if ks[p] == M64:
            continue
        for q in range(1, win + 1):
            if p + q >= len(ks) or ks[p + q] != ks[p]:
                break
            a, c = it[p], it[p + q]
            pairs.add((min(a, c), max(a, c)))
    return sorted(pairs)


def jaccard(a, b):
    if len(a) == 0 or len(b) == 0:
        return 0.0
    sa, sb = set(a), set(b)
    inter = len(sa & sb)
    return inter / (len(sa) + len(sb) - inter)


def greedy_merge(sets, pairs, cap):
    n = len(sets)
    parent = list(range(n))
    size = [1] * n
    deleted = [False] * n

    def root(i):
        while i != parent[i]:
            parent[i] = parent[parent[i]]
            i = parent[i]
        return i

    heap = [(-jaccard(sets[a], sets[b]), a, b) for a, b in pairs]
    heapq.heapify(heap)
    queued = set(pairs)
    num_cluster = n
    while heap and num_cluster > 0:
        _, p1, p2 = heapq.heappop(heap)
        queued.discard((min(p1, p2), max(p1, p2)))
        if p1 == parent[p1] and p2 == parent[p2]:
            if deleted[p1] or deleted[p2]:
                continue
            if size[p1] < size[p2]:
                parent[p1] = p2
                num_cluster -= 1
                size[p2] += size[p1]
                if size[p2] >= cap:
                    deleted[p2] = True
                    num_cluster -= 1
            else:
                parent[p2] = p1
                num_cluster -= 1
                size[p1] += size[p2]
                if size[p1] >= cap:
                    deleted[p1] = True
                    num_cluster -= 1
        else:
            p1, p2 = root(p1), root(p2)
            if deleted[p1] or deleted[p2]:
                continue
            k = (min(p1, p2), max(p1, p2))
            if p1 != p2 and k not in queued:
                heapq.heappush(heap, (-jaccard(sets[p1], sets[p2]), p1, p2))
                queued.add(k)
    return [root(i) for i in range(n)]


def groups_of(roots):
    gid, groups = {}, []
    for i, r in enumerate(roots):
        if r not in gid:
            gid[r] = len(groups)
            groups.append([])
        groups[gid[r]].append(i)
    return groups


def two_level(rows, pairs1, pairs2_of, thres, c_thres):
    """The two clustering levels and the output order (TCA_reorder.py:154-307).

    rows: the rows' column sets; pairs1: level-1 candidate pairs (lo, hi);
    pairs2_of(g1, csets): level-2 candidate pairs over the level-1 clusters g1
    (in order of first appearance) whose column sets are csets (the union of
    their rows' sets). The candidate rule is the caller's: the library's LSH
    (tca_perm) or any other rule fed to the reference's own merge."""
    g1 = groups_of(greedy_merge(rows, pairs1, thres))
    csets = [np.unique(np.concatenate([np.asarray(rows[i], np.int64) for i in g])) for g in g1]
    g2 = groups_of(greedy_merge(csets, pairs2_of(g1, csets), c_thres))
    return np.array([row for g in g2 for c in g for row in g1[c]], np.int32)


def threshold_pairs(sets, thr):
    """Pairs (lo, hi) of nonempty sets whose exact Jaccard is >= thr: an
    exact stand-in for MinHash LSH at threshold thr."""
    n = len(sets)
    ss = [set(int(x) for x in s) for s in sets]
    out = []
    for a in range(n):
        if not ss[a]:
            continue
        for b in range(a + 1, n):
            if ss[b]:
                inter = len(ss[a] & ss[b])
                if inter / len(ss[a] | ss[b]) >= thr:
                    out.append((a, b))
    return out


def tca_perm(rowptr, col, M, **params):
    p = dict(DEFAULTS, **params)
    rowptr = np.asarray(rowptr, np.int64)
    col = np.asarray(col, np.int64)
    rows = [np.unique(col[rowptr[i]:rowptr[i + 1]]) for i in range(M)]
    P, b, r, w = p["num_perm"], p["bands"], p["rows_per_band"], p["bucket_window"]
    rsig = signatures(rows, P, p["seed"])

    def pairs2_of(g1, csets):
        csig = np.stack([rsig[g].min(axis=0) for g in g1]).astype(np.uint32)
        return lsh_pairs(csig, b, r, w)
    return two_level(rows, lsh_pairs(rsig, b, r, w), pairs2_of, p["thres"], p["c_thres"])
