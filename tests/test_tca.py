"""TCA reorder (reordering/TCA_reorder.py:53-326): the library's permutation is
bit-exact with the oracle's restatement (same hashing, banding and merge
rules), is a permutation, respects the level-1 cluster cap, and reduces the
ME-TCF block count on a matrix with hidden row clusters. The oracle's merge,
level-2 clustering and output order are pinned to the reference script's own
run (tests/golden/ref_tca_*.npz, made by tests/golden/make_tca_golden.py with
exact-threshold candidates in place of MinHash LSH)."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from oracle import tca_oracle as TO


def clustered(M=480, groups=30, seed=0):
    """Rows in hidden groups sharing column sets, shuffled over the row ids."""
    rng = np.random.default_rng(seed)
    pool = [rng.choice(M, 12, replace=False) for _ in range(groups)]
    owner = rng.permutation(np.arange(M) % groups)
    rows = []
    for i in range(M):
        base = pool[owner[i]]
        keep = base[rng.random(len(base)) < 0.85]
        extra = rng.choice(M, 1)
        rows.append(np.unique(np.concatenate([keep, extra])))
    rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int32)
    return rp, np.concatenate(rows).astype(np.int32), M


def test_oracle_clusters_respect_caps():
    rp, col, M = clustered(M=200, groups=10)
    perm = TO.tca_perm(rp, col, M, thres=16)
    assert sorted(perm.tolist()) == list(range(M))
    rows = [np.unique(col[rp[i]:rp[i + 1]]) for i in range(M)]
    sig = TO.signatures(rows, 128, 2022)
    roots = TO.greedy_merge(rows, TO.lsh_pairs(sig, 42, 3, 8), 16)
    sizes = np.bincount(roots)
    # a cluster stops growing once it reaches the cap; the last merge can overshoot
    assert sizes.max() < 2 * 16


TCA_GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "ref_tca_*.npz")))
LSH_THRES = 0.2      # lsh_thres and cluster_thres of the script (TCA_reorder.py:21-23)
C_THRES = 128        # c_thres (TCA_reorder.py:22)


def test_tca_golden_present():
    assert len(TCA_GOLDEN) >= 6


@pytest.mark.parametrize("path", TCA_GOLDEN, ids=lambda p: os.path.basename(p)[8:-4])
def test_oracle_merge_matches_reference_script(path):
    """Same candidate pairs (exact Jaccard >= 0.2 at both levels, the rule the
    script's MinHash LSH approximates) -> the reference's reorder_id, bit for
    bit: merge order and direction, the cluster cap, requeues of roots with
    their own sets, level-2 clustering at cap 128 and the output order."""
    z = np.load(path)
    n, src, dst = int(z["num_nodes"]), z["src_li"], z["dst_li"]
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    rp = np.searchsorted(src, np.arange(n + 1)).astype(np.int64)
    rows = [np.unique(dst[rp[i]:rp[i + 1]]) for i in range(n)]
    assert all(len(r) for r in rows)
    assert int(z["ties"][0]) > 0  # the tie rule is exercised
    perm = TO.two_level(rows, TO.threshold_pairs(rows, LSH_THRES),
                        lambda g1, csets: TO.threshold_pairs(csets, LSH_THRES),
                        int(z["thres"]), C_THRES)
    np.testing.assert_array_equal(perm, z["reorder_id"])


def _golden_csr(z):
    n, src, dst = int(z["num_nodes"]), z["src_li"], z["dst_li"]
    order = np.lexsort((dst, src))
    src, dst = src[order], dst[order]
    return np.searchsorted(src, np.arange(n + 1)).astype(np.int32), dst.astype(np.int32), n


@pytest.mark.parametrize("path", TCA_GOLDEN, ids=lambda p: os.path.basename(p)[8:-4])
def test_oracle_relabel_matches_reference_pipeline(path):
    """P A P^T with the script's reorder_id equals the reference pipeline's
    reordered CSR: its relabelled edge list (TCA_reorder.py:316-326) read by
    its graph loader (scripts/DTCSpMM/dataset.py:21-44)."""
    z = np.load(path)
    rp, col, n = _golden_csr(z)
    orp, oc, _ = O.permute_csr(rp, col, None, z["reorder_id"].astype(np.int64))
    np.testing.assert_array_equal(orp, z["reordered_row_pointers"])
    np.testing.assert_array_equal(oc, z["reordered_column_index"])


@pytest.mark.gpu
@pytest.mark.parametrize("path", TCA_GOLDEN, ids=lambda p: os.path.basename(p)[8:-4])
def test_permute_matches_reference_pipeline(cuda, path):
    import torch
    from dtc_b200 import metcf
    z = np.load(path)
    rp, col, n = _golden_csr(z)
    g = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    grp, gc, _ = metcf.permute_csr(g(rp), g(col), None, g(z["reorder_id"].astype(np.int32)))
    np.testing.assert_array_equal(grp.cpu().numpy(), z["reordered_row_pointers"])
    np.testing.assert_array_equal(gc.cpu().numpy(), z["reordered_column_index"])


@pytest.mark.parametrize("path", TCA_GOLDEN, ids=lambda p: os.path.basename(p)[8:-4])
def test_library_merge_matches_reference_script(path):
    """The library's host clustering (reorder.cluster_order: both levels on
    dtc_tca_merge, the greedy_merge that dtc_tca_reorder runs; no GPU)
    reproduces the reference script's reorder_id from the same candidates."""
    from dtc_b200 import reorder
    z = np.load(path)
    rp, col, n = _golden_csr(z)
    rows = [np.unique(col[rp[i]:rp[i + 1]]) for i in range(n)]
    got = reorder.cluster_order(rows, lambda sets: TO.threshold_pairs(sets, LSH_THRES),
                                int(z["thres"]), C_THRES)
    np.testing.assert_array_equal(got, z["reorder_id"])


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_library_merge_matches_oracle_on_lsh_pairs(seed):
    """Same roots as the oracle's greedy_merge on the library's LSH candidate
    rule (many equal scores, requeues, both caps)."""
    from dtc_b200 import reorder
    rp, col, M = clustered(M=300, groups=20, seed=seed)
    rows = [np.unique(col[rp[i]:rp[i + 1]]) for i in range(M)]
    pairs = TO.lsh_pairs(TO.signatures(rows, 128, 2022), 42, 3, 8)
    for cap in (2, 4, 16):
        np.testing.assert_array_equal(reorder.merge_pairs(rows, pairs, cap),
                                      TO.greedy_merge(rows, pairs, cap))


@pytest.mark.parametrize("seed", [0, 1])
def test_cluster_order_with_lsh_rule_is_tca_perm(seed):
    """cluster_order on the library's LSH candidate rule is the oracle's
    tca_perm (which dtc_tca_reorder equals bit for bit on the GPU): at level 2
    the signature of a cluster's union is the min of its rows' signatures."""
    from dtc_b200 import reorder
    rp, col, M = clustered(M=320, groups=24, seed=seed)
    rows = [np.unique(col[rp[i]:rp[i + 1]]) for i in range(M)]
    rule = lambda sets: TO.lsh_pairs(TO.signatures(sets, 128, 2022), 42, 3, 8)
    np.testing.assert_array_equal(reorder.cluster_order(rows, rule, 8, 16),
                                  TO.tca_perm(rp, col, M, thres=8, c_thres=16))


@pytest.mark.parametrize("seed", range(6))
def test_library_merge_matches_oracle_fuzz(seed):
    """Random small sets (some empty, many overlapping) and random candidate
    pairs: equal and zero scores everywhere, requeues and caps from 1 to 8;
    the library's roots equal the oracle's."""
    from dtc_b200 import reorder
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(2, 80))
    sets = [np.unique(rng.integers(0, 12, int(rng.integers(0, 6)))) for _ in range(n)]
    m = int(rng.integers(0, 4 * n))
    pairs = sorted({(int(min(a, b)), int(max(a, b)))
                    for a, b in rng.integers(0, n, (m, 2)) if a != b})
    for cap in (1, 2, 3, 8):
        np.testing.assert_array_equal(reorder.merge_pairs(sets, pairs, cap),
                                      TO.greedy_merge(sets, pairs, cap))


def test_library_merge_accepts_csr_sets():
    from dtc_b200 import _lib, reorder
    rp, col, M = clustered(M=200, groups=12, seed=5)
    rows = [np.unique(col[rp[i]:rp[i + 1]]) for i in range(M)]
    ptr = np.concatenate([[0], np.cumsum([len(r) for r in rows])])
    idx = np.concatenate(rows)
    pairs = TO.lsh_pairs(TO.signatures(rows, 128, 2022), 42, 3, 8)
    np.testing.assert_array_equal(reorder.merge_pairs((ptr, idx), pairs, 8),
                                  reorder.merge_pairs(rows, pairs, 8))
    with pytest.raises(_lib.DtcError):  # rows must be sorted and distinct
        reorder.merge_pairs((np.array([0, 2]), np.array([3, 1])), [], 4)


def test_library_merge_rejects_bad_input():
    from dtc_b200 import _lib, reorder
    rows = [np.array([0, 1]), np.array([1, 2]), np.array([5])]
    with pytest.raises(_lib.DtcError):
        reorder.merge_pairs(rows, [(1, 0)], 4)          # lo > hi
    with pytest.raises(_lib.DtcError):
        reorder.merge_pairs(rows, [(0, 3)], 4)          # hi out of range
    with pytest.raises(_lib.DtcError):
        reorder.merge_pairs(rows, [(0, 1)], 0)          # cap < 1
    assert reorder.merge_pairs([], [], 4).shape == (0,)
    np.testing.assert_array_equal(reorder.merge_pairs(rows, [], 4), [0, 1, 2])


def test_oracle_mix64_matches_vectorised():
    xs = [0, 1, 2 ** 63 + 5, 123456789]
    np.testing.assert_array_equal(TO._mix64_np(np.array(xs, np.uint64)),
                                  np.array([TO._mix64(x) for x in xs], np.uint64))


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1])
def test_tca_perm_bit_exact(cuda, seed):
    import torch
    from dtc_b200 import reorder
    rp, col, M = clustered(seed=seed)
    got = reorder.tca_perm(torch.from_numpy(rp).cuda(), torch.from_numpy(col).cuda(), M)
    ref = TO.tca_perm(rp, col, M)
    np.testing.assert_array_equal(got.cpu().numpy(), ref)


@pytest.mark.gpu
def test_tca_perm_with_empty_rows_and_hub(cuda):
    import torch
    from dtc_b200 import reorder
    from tests.golden import cases
    rp, col, _, M = cases.hub()
    got = reorder.tca_perm(torch.from_numpy(rp).cuda(), torch.from_numpy(col).cuda(), M,
                           reorder.default_params(thres=8, c_thres=16))
    ref = TO.tca_perm(rp, col, M, thres=8, c_thres=16)
    np.testing.assert_array_equal(got.cpu().numpy(), ref)


@pytest.mark.gpu
def test_tca_reduces_blocks_on_hidden_clusters(cuda):
    import torch
    from dtc_b200 import metcf, reorder
    rp, col, M = clustered(M=2048, groups=128, seed=3)
    rpd, cd = torch.from_numpy(rp).cuda(), torch.from_numpy(col).cuda()
    T0 = metcf.convert(rpd, cd, M).T
    perm, rp2, c2, _ = reorder.reorder(rpd, cd, None, M)
    T1 = metcf.convert(rp2, c2, M).T
    assert sorted(perm.cpu().tolist()) == list(range(M))
    assert T1 < 0.8 * T0, (T0, T1)
