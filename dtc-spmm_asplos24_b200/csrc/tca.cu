// TCA reorder: two-level MinHash-LSH + Jaccard clustering of rows
// (reordering/TCA_reorder.py:53-326), producing the permutation that packs
// rows with similar column sets into the same row windows.
//
// Level 1 ("TCU-aware", :53-241): rows are items, each with its column set.
// Level 2 ("cache-aware", :243-305): the level-1 clusters are items, each with
// the union of its rows' column sets. At each level:
//   1. MinHash signatures, `num_perm` hash functions (GPU; a cluster's
//      signature is the element-wise min of its rows' signatures, which is the
//      MinHash of the union).
//   2. LSH banding: `bands` bands of `rows_per_band` signature values; items
//      whose band values all agree share a bucket (GPU radix sort of
//      (band, band-hash) keys). Each item is paired with the next
//      `bucket_window` items of its bucket (the reference pairs every bucket
//      member; the window bounds hub buckets).
//   3. Exact Jaccard similarity of every distinct candidate pair (GPU, one
//      thread per pair merging the two sorted sets), then a stable radix sort
//      of the pairs by descending similarity (ties keep the (first, second)
//      order of the sorted pair list).
//   4. Greedy merging by descending similarity with union-find, exactly the
//      reference's loop (:171-205 / :268-293): two live roots merge (smaller
//      size into larger; ties into the first of the pair); a cluster whose
//      size reaches the cap (`thres` rows at level 1, `c_thres` clusters at
//      level 2) stops merging; a pair whose ends are no longer roots is
//      requeued once as (root, root) with the Jaccard of the two roots' own
//      item sets. Ties in similarity pop in (first, second) order. The loop
//      walks the sorted initial pairs and keeps only requeued pairs in a heap.
// Clusters are numbered in order of their smallest member, members ascending;
// the output lists level-2 groups in that order, each group's clusters in
// ascending number and each cluster's rows ascending (:308-315).
// Items with an empty set never enter LSH and stay singletons.
#include <cub/cub.cuh>
#include <algorithm>
#include <new>
#include <queue>
#include <vector>
#include "common.cuh"

namespace dtc {
namespace {

constexpr int kThreads = 256;

inline unsigned grid_for(int64_t n) {
  int64_t g = (n + kThreads - 1) / kThreads;
  if (g < 1) g = 1;
  if (g > (1 << 30)) g = 1 << 30;
  return (unsigned)g;
}

// splitmix64 finaliser (Steele, Lea, Flood 2014): a bijective 64-bit mixer.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// sig[i * P + k] = min over columns c of row i of h_k(c), where h_k(c) is the
// high 32 bits of mix64(c ^ salt_k), salt_k = mix64(seed + 0x9e37...15 * (k+1));
// rows without columns keep 0xffffffff. One warp per row, lanes over k.
__global__ void k_row_signatures(const int32_t* __restrict__ rowptr,
                                 const int32_t* __restrict__ col, int32_t M, int P,
                                 uint64_t seed, uint32_t* __restrict__ sig) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < M; r += nwarps) {
    const int32_t e0 = rowptr[r], e1 = rowptr[r + 1];
    for (int k = lane; k < P; k += 32) {
      uint64_t salt = mix64(seed + 0x9e3779b97f4a7c15ull * (uint64_t)(k + 1));
      uint32_t m = 0xffffffffu;
      for (int32_t e = e0; e < e1; ++e) {
        const uint32_t h = (uint32_t)(mix64((uint64_t)(uint32_t)col[e] ^ salt) >> 32);
        m = h < m ? h : m;
      }
      sig[r * P + k] = m;
    }
  }
}

// Cluster signatures: element-wise min over member rows (cid[row] = cluster).
__global__ void k_cluster_signatures(const uint32_t* __restrict__ rsig,
                                     const int32_t* __restrict__ cid, int32_t M, int P,
                                     uint32_t* __restrict__ csig) {
  const int64_t n = (int64_t)M * P;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t r = (int32_t)(i / P);
    const int k = (int)(i % P);
    const uint32_t v = rsig[i];
    if (v != 0xffffffffu) atomicMin(csig + (int64_t)cid[r] * P + k, v);
  }
}

// Band keys: key = band << 40 | 40 bits of the hash of the band's values.
// Items with an empty set get the sentinel key ~0 (sorted last, never paired).
__global__ void k_band_keys(const uint32_t* __restrict__ sig, int32_t n, int P, int bands,
                            int rpb, uint64_t* __restrict__ keys, int32_t* __restrict__ items) {
  const int64_t total = (int64_t)n * bands;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += stride) {
    const int b = (int)(t / n);
    const int32_t i = (int32_t)(t % n);
    const uint32_t* s = sig + (int64_t)i * P + b * rpb;
    uint64_t h = 0x51ed27a3c0ffee11ull ^ (uint64_t)b;
    bool empty = false;
    for (int j = 0; j < rpb; ++j) {
      empty |= (s[j] == 0xffffffffu);
      h = mix64(h ^ s[j]);
    }
    keys[t] = empty ? ~0ull : (((uint64_t)b << 40) | (h & ((1ull << 40) - 1)));
    items[t] = i;
  }
}

// Pairs of each sorted position with the next `win` positions of its bucket:
// pass 0 counts, pass 1 writes (lo << 32 | hi) at the scanned offsets.
__global__ void k_bucket_pairs(const uint64_t* __restrict__ keys, const int32_t* __restrict__ items,
                               int64_t n, int win, int32_t* __restrict__ counts,
                               const int32_t* __restrict__ offs, uint64_t* __restrict__ pairs) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < n; p += stride) {
    const uint64_t k = keys[p];
    int c = 0;
    if (k != ~0ull) {
      for (int q = 1; q <= win && p + q < n && keys[p + q] == k; ++q) {
        if (pairs) {
          uint32_t a = (uint32_t)items[p], b = (uint32_t)items[p + q];
          if (a > b) { uint32_t t = a; a = b; b = t; }
          pairs[offs[p] + c] = ((uint64_t)a << 32) | b;
        }
        ++c;
      }
    }
    if (!pairs) counts[p] = c;
  }
}

// score[i] = Jaccard of the sorted, distinct sets of the two items of pair i
// (hi << 32 | lo packing: lo < hi), exactly (double)|a ∩ b| / |a ∪ b| as the
// host computes it; 0 when either set is empty.
__global__ void k_pair_jaccard(const uint64_t* __restrict__ pairs, int64_t np,
                               const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                               double* __restrict__ score) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < np; i += stride) {
    const uint64_t pr = pairs[i];
    const int32_t a = (int32_t)(pr >> 32), b = (int32_t)(pr & 0xffffffffu);
    int64_t ia = ptr[a], ea = ptr[a + 1], ib = ptr[b], eb = ptr[b + 1];
    const int64_t na = ea - ia, nb = eb - ib;
    double s = 0.0;
    if (na > 0 && nb > 0) {
      int64_t inter = 0;
      int32_t va = idx[ia], vb = idx[ib];
      while (true) {
        if (va < vb) {
          if (++ia == ea) break;
          va = idx[ia];
        } else if (va > vb) {
          if (++ib == eb) break;
          vb = idx[ib];
        } else {
          ++inter;
          if (++ia == ea || ++ib == eb) break;
          va = idx[ia];
          vb = idx[ib];
        }
      }
      s = (double)inter / (double)(na + nb - inter);
    }
    score[i] = s;
  }
}

// Device workspace for one level over n items with P-value signatures.
// Workspace of one banding + scoring pass. The distinct pair keys (pairs_in)
// live through both stages; the banding stage's buffers (band keys, raw pairs,
// their sort) are dead once the distinct pairs are known, so the scoring stage
// (scores, order, its sort) reuses the same bytes: the pass needs the larger
// stage, not their sum.
struct LshLayout {
  size_t keys_in, keys_out, items_in, items_out, counts, offs, pairs_in, pairs_out, sort1, scan,
      sort2, uniq, uniq_bytes, nsel, score_in, score_out, ord_in, ord_out, sort3, sort3_bytes, total;
};

// skey[j] = keys[ord[j]] (the pairs in score order) and rank[ord[j]] = j (the
// position of keys[i] in that order).
__global__ void k_score_order(const uint64_t* __restrict__ keys, const int32_t* __restrict__ ord,
                              int64_t n, uint64_t* __restrict__ skey, int32_t* __restrict__ rank) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += stride) {
    const int32_t o = ord[j];
    skey[j] = keys[o];
    rank[o] = (int32_t)j;
  }
}

// keys[e] = (cid[r] << 32) | member e of item r's set (one warp per item).
__global__ void k_cluster_keys(const int64_t* __restrict__ ptr, const int32_t* __restrict__ idx,
                               const int32_t* __restrict__ cid, int32_t n,
                               uint64_t* __restrict__ keys) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < n; r += nwarps) {
    const uint64_t hi = (uint64_t)(uint32_t)cid[r] << 32;
    for (int64_t e = ptr[r] + lane; e < ptr[r + 1]; e += 32) keys[e] = hi | (uint32_t)idx[e];
  }
}

// CSR of the sorted distinct (cluster, member) keys: ptr[c] = first key of
// cluster c (binary search), idx[i] = member of key i.
__global__ void k_cluster_csr(const uint64_t* __restrict__ keys, int64_t nk, int32_t nc,
                              int64_t* __restrict__ ptr, int32_t* __restrict__ idx) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nk; i += stride)
    idx[i] = (int32_t)(keys[i] & 0xffffffffu);
  for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c <= nc; c += stride) {
    const uint64_t key = (uint64_t)(uint32_t)c << 32;
    int64_t lo = 0, hi = nk;
    while (lo < hi) {
      const int64_t mid = (lo + hi) >> 1;
      if (keys[mid] < key) lo = mid + 1; else hi = mid;
    }
    ptr[c] = lo;
  }
}

// ord[i] = i.
__global__ void k_iota(int32_t* __restrict__ ord, int64_t n) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride)
    ord[i] = (int32_t)i;
}

LshLayout lsh_layout(int64_t n_keys, int64_t max_pairs) {
  LshLayout L{};
  size_t off = 0;
  auto take = [&](size_t b) { size_t o = off; off = align_up(off + (b ? b : 1), 256); return o; };
  const size_t n = (size_t)(n_keys > 0 ? n_keys : 1);
  const size_t mp = (size_t)(max_pairs > 0 ? max_pairs : 1);
  L.pairs_in = take(mp * 8);
  L.nsel = take(8);
  const size_t stage_base = off;
  // banding stage
  L.keys_in = take(n * 8);
  L.keys_out = take(n * 8);
  L.items_in = take(n * 4);
  L.items_out = take(n * 4);
  L.counts = take((n + 1) * 4);
  L.offs = take((n + 1) * 4);
  L.pairs_out = take(mp * 8);
  size_t s1 = 0, s2 = 0, s3 = 0, s4 = 0, s5 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, s1, (uint64_t*)nullptr, (uint64_t*)nullptr,
                                  (int32_t*)nullptr, (int32_t*)nullptr, (int64_t)n);
  cub::DeviceScan::ExclusiveSum(nullptr, s2, (int32_t*)nullptr, (int32_t*)nullptr, (int64_t)n + 1);
  // (the raw pairs, and the cluster-member keys of the second level, n of them)
  const size_t ns = n > mp ? n : mp;
  cub::DeviceRadixSort::SortKeys(nullptr, s3, (uint64_t*)nullptr, (uint64_t*)nullptr, (int64_t)ns);
  cub::DeviceSelect::Unique(nullptr, s5, (uint64_t*)nullptr, (uint64_t*)nullptr,
                            (int64_t*)nullptr, (int64_t)ns);
  cub::DeviceRadixSort::SortPairsDescending(nullptr, s4, (double*)nullptr, (double*)nullptr,
                                            (int32_t*)nullptr, (int32_t*)nullptr, (int64_t)mp);
  L.sort1 = take(s1);
  L.scan = take(s2);
  L.sort2 = take(s3);
  L.uniq = take(s5);
  L.uniq_bytes = s5;
  const size_t banding_end = off;
  // scoring stage, over the banding stage's bytes
  off = stage_base;
  L.score_in = take(mp * 8);
  L.score_out = take(mp * 8);
  L.ord_in = take(mp * 4);
  L.ord_out = take(mp * 4);
  L.sort3 = take(s4);
  L.sort3_bytes = s4;
  L.total = off > banding_end ? off : banding_end;
  return L;
}

// Candidate pairs of one level: distinct (lo << 32 | hi, lo < hi) in ascending
// order, their Jaccard scores, and the order of descending score (ties in
// ascending pair order).
struct Scored {
  std::vector<uint64_t> keys;   // ascending
  std::vector<uint64_t> skey;   // the same pairs, best score first
  std::vector<double> score;    // score of skey[j]
  std::vector<int32_t> rank;    // position of keys[i] in skey
};

// Candidate pairs for n items whose sorted, distinct sets are d_ptr / d_idx
// (device CSR), scored on the GPU.
dtc_status lsh_pairs(const uint32_t* sig, int32_t n, const dtc_tca_params& prm, char* ws,
                     const LshLayout& L, int64_t max_pairs, const int64_t* d_ptr,
                     const int32_t* d_idx, cudaStream_t st, Scored& out) {
  out.keys.clear();
  out.skey.clear();
  out.score.clear();
  out.rank.clear();
  if (n < 2) return DTC_OK;
  const int64_t nk = (int64_t)n * prm.bands;
  uint64_t* kin = (uint64_t*)(ws + L.keys_in);
  uint64_t* kout = (uint64_t*)(ws + L.keys_out);
  int32_t* iin = (int32_t*)(ws + L.items_in);
  int32_t* iout = (int32_t*)(ws + L.items_out);
  int32_t* counts = (int32_t*)(ws + L.counts);
  int32_t* offs = (int32_t*)(ws + L.offs);
  uint64_t* pin = (uint64_t*)(ws + L.pairs_in);
  uint64_t* pout = (uint64_t*)(ws + L.pairs_out);
  k_band_keys<<<grid_for(nk), kThreads, 0, st>>>(sig, n, prm.num_perm, prm.bands,
                                                 prm.rows_per_band, kin, iin);
  size_t b1 = L.scan - L.sort1;
  DTC_CUDA(cub::DeviceRadixSort::SortPairs(ws + L.sort1, b1, kin, kout, iin, iout, nk, 0, 64, st));
  k_bucket_pairs<<<grid_for(nk), kThreads, 0, st>>>(kout, iout, nk, prm.bucket_window, counts,
                                                    nullptr, nullptr);
  DTC_CUDA(cudaMemsetAsync(counts + nk, 0, 4, st));
  size_t b2 = L.sort2 - L.scan;
  DTC_CUDA(cub::DeviceScan::ExclusiveSum(ws + L.scan, b2, counts, offs, nk + 1, st));
  int32_t np = 0;
  DTC_CUDA(cudaMemcpyAsync(&np, offs + nk, 4, cudaMemcpyDeviceToHost, st));
  DTC_CUDA(cudaStreamSynchronize(st));
  if (np <= 0) return DTC_OK;
  if (np > max_pairs) {
    set_error("tca: candidate pairs exceed the workspace bound");
    return DTC_ERR_WORKSPACE_TOO_SMALL;
  }
  k_bucket_pairs<<<grid_for(nk), kThreads, 0, st>>>(kout, iout, nk, prm.bucket_window, counts,
                                                    offs, pin);
  size_t b3 = L.uniq - L.sort2;
  DTC_CUDA(cub::DeviceRadixSort::SortKeys(ws + L.sort2, b3, pin, pout, (int64_t)np, 0, 64, st));
  int64_t* nsel = (int64_t*)(ws + L.nsel);
  size_t b4 = L.uniq_bytes;
  DTC_CUDA(cub::DeviceSelect::Unique(ws + L.uniq, b4, pout, pin, nsel, (int64_t)np, st));
  int64_t nu = 0;
  DTC_CUDA(cudaMemcpyAsync(&nu, nsel, 8, cudaMemcpyDeviceToHost, st));
  DTC_CUDA(cudaStreamSynchronize(st));
  double* sin = (double*)(ws + L.score_in);
  double* sout = (double*)(ws + L.score_out);
  int32_t* oin = (int32_t*)(ws + L.ord_in);
  int32_t* oout = (int32_t*)(ws + L.ord_out);
  k_pair_jaccard<<<grid_for(nu), kThreads, 0, st>>>(pin, nu, d_ptr, d_idx, sin);
  k_iota<<<grid_for(nu), kThreads, 0, st>>>(oin, nu);
  DTC_CUDA(cudaGetLastError());
  size_t b5 = L.sort3_bytes;
  DTC_CUDA(cub::DeviceRadixSort::SortPairsDescending(ws + L.sort3, b5, sin, sout, oin, oout, nu,
                                                     0, 64, st));
  // the sort's inputs are dead: score order of the keys into sin, ranks into oin
  uint64_t* skey = (uint64_t*)sin;
  int32_t* rank = oin;
  k_score_order<<<grid_for(nu), kThreads, 0, st>>>(pin, oout, nu, skey, rank);
  DTC_CUDA(cudaGetLastError());
  out.keys.resize(nu);
  out.skey.resize(nu);
  out.score.resize(nu);
  out.rank.resize(nu);
  DTC_CUDA(cudaMemcpyAsync(out.keys.data(), pin, (size_t)nu * 8, cudaMemcpyDeviceToHost, st));
  DTC_CUDA(cudaMemcpyAsync(out.skey.data(), skey, (size_t)nu * 8, cudaMemcpyDeviceToHost, st));
  DTC_CUDA(cudaMemcpyAsync(out.score.data(), sout, (size_t)nu * 8, cudaMemcpyDeviceToHost, st));
  DTC_CUDA(cudaMemcpyAsync(out.rank.data(), rank, (size_t)nu * 4, cudaMemcpyDeviceToHost, st));
  DTC_CUDA(cudaStreamSynchronize(st));
  return DTC_OK;
}

// Jaccard |a ∩ b| / |a ∪ b| of two sorted, distinct lists (0 when either is empty).
double jaccard(const int32_t* a, int64_t na, const int32_t* b, int64_t nb) {
  if (na == 0 || nb == 0) return 0.0;
  if (na > nb) {  // a is the smaller list
    std::swap(a, b);
    std::swap(na, nb);
  }
  int64_t inter = 0;
  if (na * 32 < nb) {
    // sizes far apart (a hub row against a short one): gallop through b for
    // each member of a, O(na log nb) instead of O(na + nb)
    int64_t j = 0;
    for (int64_t i = 0; i < na && j < nb; ++i) {
      const int32_t x = a[i];
      int64_t step = 1, hi = j;
      while (hi < nb && b[hi] < x) { j = hi + 1; hi += step; step <<= 1; }
      if (hi > nb) hi = nb;
      j = std::lower_bound(b + j, b + hi, x) - b;
      if (j < nb && b[j] == x) { ++inter; ++j; }
    }
  } else {
    // branchless merge: each step advances past the smaller head (both on a match)
    int64_t i = 0, j = 0;
    while (i < na && j < nb) {
      const int32_t x = a[i], y = b[j];
      inter += (x == y);
      i += (x <= y);
      j += (y <= x);
    }
  }
  return (double)inter / (double)(na + nb - inter);
}

// Item sets as CSR of sorted distinct members.
struct Sets {
  std::vector<int64_t> ptr;
  std::vector<int32_t> idx;
  double jac(int32_t a, int32_t b) const {
    return jaccard(idx.data() + ptr[a], ptr[a + 1] - ptr[a], idx.data() + ptr[b],
                   ptr[b + 1] - ptr[b]);
  }
};

// Set of pair keys (a << 32 | b, a, b < 2^31): open addressing with linear
// probing and tombstones, rehashed at half load. Holds the requeued pairs
// currently in the merge heap.
class PairSet {
 public:
  PairSet() { rehash(1024); }
  bool contains(uint64_t k) const {
    for (size_t i = slot(k);; i = (i + 1) & mask_) {
      if (t_[i] == k) return true;
      if (t_[i] == kEmpty) return false;
    }
  }
  void insert(uint64_t k) {
    if (2 * (used_ + 1) > t_.size()) rehash(live_ * 4 > 1024 ? live_ * 4 : 1024);
    size_t tomb = SIZE_MAX;
    for (size_t i = slot(k);; i = (i + 1) & mask_) {
      if (t_[i] == k) return;
      if (t_[i] == kTomb && tomb == SIZE_MAX) tomb = i;
      if (t_[i] == kEmpty) {
        if (tomb != SIZE_MAX) {
          t_[tomb] = k;
        } else {
          t_[i] = k;
          ++used_;
        }
        ++live_;
        return;
      }
    }
  }
  void erase(uint64_t k) {
    for (size_t i = slot(k);; i = (i + 1) & mask_) {
      if (t_[i] == k) {
        t_[i] = kTomb;
        --live_;
        return;
      }
      if (t_[i] == kEmpty) return;
    }
  }

 private:
  static constexpr uint64_t kEmpty = ~0ull, kTomb = ~0ull - 1;
  std::vector<uint64_t> t_;
  size_t mask_ = 0, used_ = 0, live_ = 0;  // used_: live + tombstones
  size_t slot(uint64_t k) const { return (size_t)((k * 0x9E3779B97F4A7C15ull) >> 20) & mask_; }
  void rehash(size_t want) {
    size_t cap = 1024;
    while (cap < 2 * want) cap <<= 1;
    std::vector<uint64_t> old;
    old.swap(t_);
    t_.assign(cap, kEmpty);
    mask_ = cap - 1;
    used_ = live_ = 0;
    for (uint64_t k : old)
      if (k != kEmpty && k != kTomb) insert(k);
  }
};

struct QItem {
  double s;
  int32_t a, b;
  bool operator<(const QItem& o) const {  // max-heap on s, then (a, b) ascending
    if (s != o.s) return s < o.s;
    if (a != o.a) return a > o.a;
    return b > o.b;
  }
};

// The greedy merge loop; returns the root of every item. The initial pairs
// come in score order (Scored::skey, walked front to back); requeued (root,
// root) pairs go to a heap, and the next pair is the better of the two heads
// in the QItem order.
std::vector<int32_t> greedy_merge(const Sets& sets, const Scored& sp, int32_t n, int32_t cap) {
  // Per item, packed so that one cache line serves each item the loop touches:
  // the union-find parent and the cluster size, negated once the cluster is
  // closed (the size of a closed cluster is never read again).
  struct Node {
    int32_t parent, size;
  };
  std::vector<Node> node((size_t)n);
  for (int32_t i = 0; i < n; ++i) node[i] = {i, 1};
  auto root = [&](int32_t i) {
    while (i != node[i].parent) {
      node[i].parent = node[node[i].parent].parent;
      i = node[i].parent;
    }
    return i;
  };
  auto closed = [&](int32_t i) { return node[i].size < 0; };
  auto key = [](int32_t a, int32_t b) {
    return a < b ? ((uint64_t)a << 32) | (uint32_t)b : ((uint64_t)b << 32) | (uint32_t)a;
  };
  const int64_t np = (int64_t)sp.keys.size();
  const std::vector<int32_t>& rank = sp.rank;  // position of keys[t] in the score order
  // The keys are sorted, so the initial pairs whose smaller member is a sit
  // in [first[a], first[a + 1]): the queued test searches only those.
  std::vector<int64_t> first((size_t)n + 1, 0);
  for (int64_t j = 0; j < np; ++j) ++first[(size_t)(sp.keys[j] >> 32) + 1];
  for (int32_t a = 0; a < n; ++a) first[a + 1] += first[a];
  int64_t next = 0;  // initial pairs before `next` have been popped
  std::priority_queue<QItem> q;
  PairSet requeued;  // pairs currently in the heap
  // a pair is queued when it is an initial pair not popped yet, or in the heap
  auto queued = [&](uint64_t k) {
    const size_t a = (size_t)(k >> 32);
    const auto b = sp.keys.begin() + first[a], e = sp.keys.begin() + first[a + 1];
    const auto it = std::lower_bound(b, e, k);
    if (it != e && *it == k && rank[it - sp.keys.begin()] >= next) return true;
    return requeued.contains(k);
  };
  // the initial pairs are walked in a known order: fetch the nodes of the pair
  // kAhead places further while this one is handled
  constexpr int64_t kAhead = 16;
  int64_t num_cluster = n;
  while (num_cluster > 0) {
    QItem it;
    bool from_init;
    if (next < np) {
      const uint64_t k0 = sp.skey[next];
      const QItem a{sp.score[next], (int32_t)(k0 >> 32), (int32_t)(k0 & 0xffffffffu)};
      from_init = q.empty() || !(a < q.top());
      it = from_init ? a : q.top();
    } else if (!q.empty()) {
      from_init = false;
      it = q.top();
    } else {
      break;
    }
    if (from_init) {
      if (next + kAhead < np) {
        const uint64_t kf = sp.skey[next + kAhead];
        __builtin_prefetch(&node[kf >> 32]);
        __builtin_prefetch(&node[kf & 0xffffffffu]);
        // second stage: the parents of the pair kAhead / 2 places on (their
        // nodes were fetched kAhead / 2 pops ago), the first step of root()
        const uint64_t kh = sp.skey[next + kAhead / 2];
        __builtin_prefetch(&node[node[kh >> 32].parent]);
        __builtin_prefetch(&node[node[kh & 0xffffffffu].parent]);
      }
      ++next;
    } else {
      q.pop();
      requeued.erase(key(it.a, it.b));
    }
    int32_t p1 = it.a, p2 = it.b;
    if (p1 == node[p1].parent && p2 == node[p2].parent) {
      if (closed(p1) || closed(p2)) continue;
      const int32_t s1 = node[p1].size, s2 = node[p2].size;
      --num_cluster;
      if (s1 < s2) {
        node[p1].parent = p2;
        node[p2].size = s1 + s2;
        if (s1 + s2 >= cap) { node[p2].size = -(s1 + s2); --num_cluster; }
      } else {
        node[p2].parent = p1;
        node[p1].size = s1 + s2;
        if (s1 + s2 >= cap) { node[p1].size = -(s1 + s2); --num_cluster; }
      }
    } else {
      p1 = root(p1);
      p2 = root(p2);
      if (closed(p1) || closed(p2)) continue;
      if (p1 != p2 && !queued(key(p1, p2))) {
        q.push({sets.jac(p1, p2), p1, p2});
        requeued.insert(key(p1, p2));
      }
    }
  }
  std::vector<int32_t> r(n);
  for (int32_t i = 0; i < n; ++i) r[i] = root(i);
  return r;
}

// Groups items by root in order of first appearance; members ascending.
std::vector<std::vector<int32_t>> groups_of(const std::vector<int32_t>& roots) {
  const int32_t n = (int32_t)roots.size();
  std::vector<int32_t> gid(n, -1);
  std::vector<std::vector<int32_t>> g;
  for (int32_t i = 0; i < n; ++i) {
    const int32_t r = roots[i];
    if (gid[r] < 0) { gid[r] = (int32_t)g.size(); g.emplace_back(); }
    g[gid[r]].push_back(i);
  }
  return g;
}

dtc_tca_params defaults() {
  dtc_tca_params p{};
  p.num_perm = 128;
  p.bands = 42;
  p.rows_per_band = 3;
  p.thres = 16;
  p.c_thres = 128;
  p.bucket_window = 8;
  p.seed = 2022;
  return p;
}

}  // namespace
}  // namespace dtc

using namespace dtc;

extern "C" {

void dtc_tca_default_params(dtc_tca_params* p) {
  if (p) *p = defaults();
}

dtc_status dtc_tca_workspace_bytes(int32_t num_nodes, int64_t nnz, const dtc_tca_params* params,
                                   size_t* bytes) {
  DTC_REQUIRE(bytes != nullptr, "bytes is null");
  DTC_REQUIRE(num_nodes >= 0 && nnz >= 0, "negative sizes");
  const dtc_tca_params p = params ? *params : defaults();
  DTC_REQUIRE(p.num_perm >= 1 && p.bands >= 1 && p.rows_per_band >= 1 &&
                  p.bands * p.rows_per_band <= p.num_perm,
              "need bands * rows_per_band <= num_perm");
  DTC_REQUIRE(p.bucket_window >= 1 && p.bucket_window <= 64, "bucket_window must be in [1, 64]");
  const int64_t n = num_nodes > 0 ? num_nodes : 1;
  const int64_t nk = n * p.bands;
  DTC_REQUIRE(nk * p.bucket_window < (int64_t)INT32_MAX,
              "num_nodes * bands * bucket_window must fit in int32");
  const LshLayout L = lsh_layout(nk > nnz ? nk : nnz, nk * p.bucket_window);
  size_t off = align_up((size_t)n * p.num_perm * 4, 256) * 2;  // row + cluster signatures
  off += align_up((size_t)n * 4, 256);                          // cluster id per row
  off += align_up((size_t)(n + 1) * 8, 256);                    // item sets: offsets
  off += align_up((size_t)(nnz > 0 ? nnz : 1) * 4, 256);        //            members
  *bytes = off + L.total;
  return DTC_OK;
}

dtc_status dtc_tca_reorder(const int32_t* d_rowptr, const int32_t* d_col, int32_t num_nodes,
                           int64_t nnz, const dtc_tca_params* params, int32_t* d_perm,
                           void* d_workspace, size_t workspace_bytes, dtc_stream_t stream) {
  DTC_REQUIRE(num_nodes >= 0 && nnz >= 0, "negative sizes");
  DTC_REQUIRE(d_rowptr && d_perm, "null device pointer");
  DTC_REQUIRE(nnz == 0 || d_col, "null device pointer");
  const dtc_tca_params p = params ? *params : defaults();
  DTC_REQUIRE(p.thres >= 1 && p.c_thres >= 1, "cluster caps must be >= 1");
  size_t need = 0;
  dtc_status s = dtc_tca_workspace_bytes(num_nodes, nnz, &p, &need);
  if (s != DTC_OK) return s;
  if (!d_workspace || workspace_bytes < need) {
    set_error("tca workspace too small");
    return DTC_ERR_WORKSPACE_TOO_SMALL;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const int32_t M = num_nodes;
  if (M == 0) return DTC_OK;
  // host copy of the rows' column sets (sorted, distinct)
  std::vector<int32_t> hrp(M + 1), hcol(nnz);
  DTC_CUDA(cudaMemcpyAsync(hrp.data(), d_rowptr, (size_t)(M + 1) * 4, cudaMemcpyDeviceToHost, st));
  if (nnz)
    DTC_CUDA(cudaMemcpyAsync(hcol.data(), d_col, (size_t)nnz * 4, cudaMemcpyDeviceToHost, st));
  DTC_CUDA(cudaStreamSynchronize(st));
  if (hrp[0] != 0 || hrp[M] != nnz) {
    set_error("tca: rowptr must run from 0 to nnz");
    return DTC_ERR_INVALID_ARGUMENT;
  }
  Sets rows;
  rows.ptr.resize(M + 1);
  rows.idx.reserve(nnz);
  rows.ptr[0] = 0;
  for (int32_t r = 0; r < M; ++r) {
    if (hrp[r + 1] < hrp[r]) {
      set_error("tca: rowptr must be non-decreasing");
      return DTC_ERR_INVALID_ARGUMENT;
    }
    const int32_t* b = hcol.data() + hrp[r];
    const int32_t* e = hcol.data() + hrp[r + 1];
    bool canon = true;  // sorted and distinct already (canonical CSR): no copy to sort
    for (const int32_t* x = b; x < e; ++x) {
      if (*x < 0 || *x >= M) {
        set_error("tca: column index out of range");
        return DTC_ERR_INVALID_ARGUMENT;
      }
      if (x > b && x[-1] >= *x) canon = false;
    }
    if (canon) {
      rows.idx.insert(rows.idx.end(), b, e);
    } else {
      std::vector<int32_t> v(b, e);
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
      rows.idx.insert(rows.idx.end(), v.begin(), v.end());
    }
    rows.ptr[r + 1] = (int64_t)rows.idx.size();
  }
  char* ws = (char*)d_workspace;
  const size_t sig_bytes = align_up((size_t)M * p.num_perm * 4, 256);
  uint32_t* rsig = (uint32_t*)ws;
  uint32_t* csig = (uint32_t*)(ws + sig_bytes);
  int32_t* cid = (int32_t*)(ws + 2 * sig_bytes);
  int64_t* d_set_ptr = (int64_t*)(ws + 2 * sig_bytes + align_up((size_t)M * 4, 256));
  int32_t* d_set_idx = (int32_t*)((char*)d_set_ptr + align_up((size_t)(M + 1) * 8, 256));
  char* lws = (char*)d_set_idx + align_up((size_t)(nnz > 0 ? nnz : 1) * 4, 256);
  auto upload = [&](const Sets& x) -> dtc_status {
    DTC_CUDA(cudaMemcpyAsync(d_set_ptr, x.ptr.data(), x.ptr.size() * 8, cudaMemcpyHostToDevice, st));
    if (!x.idx.empty())
      DTC_CUDA(cudaMemcpyAsync(d_set_idx, x.idx.data(), x.idx.size() * 4, cudaMemcpyHostToDevice,
                               st));
    return DTC_OK;
  };
  const int64_t nk = (int64_t)M * p.bands;
  const int64_t max_pairs = nk * p.bucket_window;
  const LshLayout L = lsh_layout(nk > nnz ? nk : nnz, max_pairs);

  // ---- level 1: rows
  k_row_signatures<<<grid_for((int64_t)M * 32), kThreads, 0, st>>>(d_rowptr, d_col, M, p.num_perm,
                                                                   p.seed, rsig);
  DTC_CUDA(cudaGetLastError());
  Scored pairs;
  s = upload(rows);
  if (s != DTC_OK) return s;
  s = lsh_pairs(rsig, M, p, lws, L, max_pairs, d_set_ptr, d_set_idx, st, pairs);
  if (s != DTC_OK) return s;
  const auto groups1 = groups_of(greedy_merge(rows, pairs, M, p.thres));
  const int32_t nc = (int32_t)groups1.size();

  // ---- level 2: clusters, each with the union of its rows' sets, built on
  // the GPU from the rows' sets (still in d_set_ptr / d_set_idx) by sorting
  // (cluster, member) keys in the banding stage's bytes (dead between levels)
  std::vector<int32_t> hcid(M);
  for (int32_t c = 0; c < nc; ++c)
    for (int32_t r : groups1[c]) hcid[r] = c;
  DTC_CUDA(cudaMemcpyAsync(cid, hcid.data(), (size_t)M * 4, cudaMemcpyHostToDevice, st));
  DTC_CUDA(cudaMemsetAsync(csig, 0xff, (size_t)nc * p.num_perm * 4, st));
  k_cluster_signatures<<<grid_for((int64_t)M * p.num_perm), kThreads, 0, st>>>(rsig, cid, M,
                                                                              p.num_perm, csig);
  DTC_CUDA(cudaGetLastError());
  Sets cl;
  cl.ptr.assign((size_t)nc + 1, 0);
  {
    const int64_t nm = rows.ptr[M];  // members over all rows
    uint64_t* kin = (uint64_t*)(lws + L.keys_in);
    uint64_t* kout = (uint64_t*)(lws + L.keys_out);
    int64_t* nsel = (int64_t*)(lws + L.nsel);
    int64_t nu = 0;
    if (nm > 0) {
      k_cluster_keys<<<grid_for((int64_t)M * 32), kThreads, 0, st>>>(d_set_ptr, d_set_idx, cid, M,
                                                                      kin);
      DTC_CUDA(cudaGetLastError());
      size_t b3 = L.uniq - L.sort2;
      DTC_CUDA(cub::DeviceRadixSort::SortKeys(lws + L.sort2, b3, kin, kout, nm, 0, 64, st));
      size_t b4 = L.uniq_bytes;
      DTC_CUDA(cub::DeviceSelect::Unique(lws + L.uniq, b4, kout, kin, nsel, nm, st));
      DTC_CUDA(cudaMemcpyAsync(&nu, nsel, 8, cudaMemcpyDeviceToHost, st));
      DTC_CUDA(cudaStreamSynchronize(st));
    }
    k_cluster_csr<<<grid_for((nu > nc ? nu : nc) + 1), kThreads, 0, st>>>(kin, nu, nc, d_set_ptr,
                                                                         d_set_idx);
    DTC_CUDA(cudaGetLastError());
    cl.idx.resize((size_t)nu);
    DTC_CUDA(cudaMemcpyAsync(cl.ptr.data(), d_set_ptr, ((size_t)nc + 1) * 8,
                             cudaMemcpyDeviceToHost, st));
    if (nu > 0)
      DTC_CUDA(cudaMemcpyAsync(cl.idx.data(), d_set_idx, (size_t)nu * 4, cudaMemcpyDeviceToHost,
                               st));
    DTC_CUDA(cudaStreamSynchronize(st));
  }
  s = lsh_pairs(csig, nc, p, lws, L, max_pairs, d_set_ptr, d_set_idx, st, pairs);
  if (s != DTC_OK) return s;
  const auto groups2 = groups_of(greedy_merge(cl, pairs, nc, p.c_thres));

  std::vector<int32_t> perm;
  perm.reserve(M);
  for (const auto& g : groups2)
    for (int32_t c : g)
      for (int32_t r : groups1[c]) perm.push_back(r);
  DTC_CUDA(cudaMemcpyAsync(d_perm, perm.data(), (size_t)M * 4, cudaMemcpyHostToDevice, st));
  DTC_CUDA(cudaStreamSynchronize(st));
  return DTC_OK;
}

}  // extern "C"

namespace {

// The body of dtc_tca_merge (host memory throughout; no CUDA call).
dtc_status merge_host(const int64_t* set_ptr, const int32_t* set_idx, int32_t n,
                      const uint64_t* pairs, int64_t num_pairs, int32_t cap, int32_t* roots) {
  DTC_REQUIRE(n >= 0 && num_pairs >= 0, "negative sizes");
  DTC_REQUIRE(num_pairs < (int64_t)INT32_MAX, "num_pairs must fit in int32");
  DTC_REQUIRE(cap >= 1, "cap must be at least 1");
  DTC_REQUIRE(n == 0 || (set_ptr && roots), "null host pointer");
  DTC_REQUIRE(num_pairs == 0 || pairs, "null host pointer");
  if (n == 0) return DTC_OK;
  Sets sets;
  sets.ptr.assign(set_ptr, set_ptr + (size_t)n + 1);
  DTC_REQUIRE(sets.ptr[0] == 0, "set_ptr[0] must be 0");
  for (int32_t i = 0; i < n; ++i)
    DTC_REQUIRE(sets.ptr[i + 1] >= sets.ptr[i], "set_ptr must be non-decreasing");
  const int64_t total = sets.ptr[n];
  DTC_REQUIRE(total == 0 || set_idx, "null host pointer");
  sets.idx.assign(set_idx, set_idx + total);
  for (int32_t i = 0; i < n; ++i)
    for (int64_t e = sets.ptr[i] + 1; e < sets.ptr[i + 1]; ++e)
      DTC_REQUIRE(sets.idx[e - 1] < sets.idx[e], "every set must be sorted and distinct");
  // the hand-over of lsh_pairs: distinct keys ascending, then the score order
  // (descending Jaccard, ties in ascending pair order) and each key's rank in it
  Scored sp;
  sp.keys.assign(pairs, pairs + num_pairs);
  for (uint64_t k : sp.keys)
    DTC_REQUIRE((k >> 32) < (k & 0xffffffffu) && (k & 0xffffffffu) < (uint64_t)n,
                "pairs must be lo << 32 | hi with lo < hi < num_items");
  std::sort(sp.keys.begin(), sp.keys.end());
  sp.keys.erase(std::unique(sp.keys.begin(), sp.keys.end()), sp.keys.end());
  const int64_t np = (int64_t)sp.keys.size();
  std::vector<double> s((size_t)np);
  for (int64_t j = 0; j < np; ++j)
    s[j] = sets.jac((int32_t)(sp.keys[j] >> 32), (int32_t)(sp.keys[j] & 0xffffffffu));
  std::vector<int64_t> order((size_t)np);
  for (int64_t j = 0; j < np; ++j) order[j] = j;
  std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) { return s[x] > s[y]; });
  sp.skey.resize(np);
  sp.score.resize(np);
  sp.rank.resize(np);
  for (int64_t r = 0; r < np; ++r) {
    sp.skey[r] = sp.keys[order[r]];
    sp.score[r] = s[order[r]];
    sp.rank[order[r]] = (int32_t)r;
  }
  const std::vector<int32_t> r = greedy_merge(sets, sp, n, cap);
  std::copy(r.begin(), r.end(), roots);
  return DTC_OK;
}

}  // namespace

extern "C" dtc_status dtc_tca_merge(const int64_t* set_ptr, const int32_t* set_idx,
                                    int32_t num_items, const uint64_t* pairs, int64_t num_pairs,
                                    int32_t cap, int32_t* roots) {
  try {
    return merge_host(set_ptr, set_idx, num_items, pairs, num_pairs, cap, roots);
  } catch (const std::bad_alloc&) {
    set_error("dtc_tca_merge: out of host memory");
    return DTC_ERR_INVALID_ARGUMENT;
  }
}
