// CSR relabelling on the GPU: symmetric row/column permutation (applying a
// TCA-style reorder) and transposition (the Aᵀ operand of a backward SpMM).
//
// The reference applies a reorder in Python (reordering/TCA_reorder.py:308-326:
// reorder[i_new] = i_old, d[old] = new, src' = d[src], dst' = d[dst]) and
// rebuilds CSR with scipy (scripts/DTCSpMM/dataset.py:38-44: coo_matrix(...)
// .tocsr(), which sorts the columns of each row and sums duplicate entries).
// Both operations here produce that canonical CSR: every edge (r, c, v) is
// mapped to (r', c'), pairs are radix-sorted by (r', c') with a stable sort,
// equal pairs are merged by summing their values in input CSR order, and the
// row pointer is rebuilt from the sorted rows.
#include <cub/cub.cuh>
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

inline int bits_for(uint64_t n) {
  int b = 0;
  while (b < 63 && (1ull << b) < n) ++b;
  return b < 1 ? 1 : b;
}

// inv[perm[i]] = i; marks bad[0] when perm is not a permutation of [0, M).
__global__ void k_invert(const int32_t* __restrict__ perm, int32_t M, int32_t* __restrict__ inv,
                         int32_t* __restrict__ seen, uint32_t* bad) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < M; i += stride) {
    const int32_t o = perm[i];
    if (o < 0 || o >= M) { atomicOr(bad, 1u); continue; }
    if (atomicAdd(seen + o, 1) != 0) { atomicOr(bad, 1u); continue; }
    inv[o] = (int32_t)i;
  }
}

// Checks the input CSR (rowptr[0] == 0, non-decreasing, rowptr[M] == nnz,
// 0 <= col < K) and writes the old row of every edge. Edge-parallel: thread e
// finds its row by binary search, the last r in [0, M) with rowptr[r] <= e
// (for a valid CSR the row holding e; empty rows before it share its start and
// lose to it). Neighbouring edges take the same search path, so a warp's loads
// are mostly broadcasts of cached entries, and a hub row of tens of thousands
// of entries costs no more than as many short rows (with a warp per row, one
// warp would walk each hub row alone). Every probe reads rowptr[1 .. M-1], so
// an invalid CSR stays in bounds; it sets the error bit and is rejected by the
// host before erow is read.
__global__ void k_rows(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                       int32_t M, int32_t K, int64_t nnz, int32_t* __restrict__ erow,
                       uint32_t* bad) {
  const int64_t t0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = t0; r < M; r += stride) {
    const int32_t e0 = __ldg(rowptr + r), e1 = __ldg(rowptr + r + 1);
    if (e1 < e0 || (r == 0 && e0 != 0) || (r == M - 1 && e1 != nnz)) atomicOr(bad, 2u);
  }
  for (int64_t e = t0; e < nnz; e += stride) {
    int32_t lo = 0, hi = M;  // rowptr[lo] <= e (rowptr[0] == 0), and hi == M or rowptr[hi] > e
    while (hi - lo > 1) {
      const int32_t mid = lo + ((hi - lo) >> 1);
      if (__ldg(rowptr + mid) <= e) lo = mid; else hi = mid;
    }
    erow[e] = lo;
    const int32_t c = __ldg(col + e);
    if (c < 0 || c >= K) atomicOr(bad, 2u);
  }
}

// COO input: erow = src, with both coordinates checked against the shape.
__global__ void k_coo_rows(const int32_t* __restrict__ src, const int32_t* __restrict__ dst,
                           int32_t M, int32_t K, int64_t nnz, int32_t* __restrict__ erow,
                           uint32_t* bad) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += stride) {
    const int32_t r = src[e], c = dst[e];
    if (r < 0 || r >= M || c < 0 || c >= K) atomicOr(bad, 2u);
    erow[e] = r;
  }
}

// key = new_row << colbits | new_col. mode 0: permutation (inv applied to
// row and column), mode 1: transpose, mode 2: identity (COO input).
__global__ void k_keys(const int32_t* __restrict__ erow, const int32_t* __restrict__ col,
                       const int32_t* __restrict__ inv, int64_t nnz, int mode, int colbits,
                       int32_t M, int32_t K, uint64_t* __restrict__ keys,
                       int32_t* __restrict__ ids) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += stride) {
    int32_t r = erow[e], c = col[e];
    r = r < 0 ? 0 : (r >= M ? M - 1 : r);   // inputs were checked; clamp keeps
    c = c < 0 ? 0 : (c >= K ? K - 1 : c);   // a bad input in bounds until the error is read
    uint64_t nr, nc;
    if (mode == 0) { nr = (uint32_t)inv[r]; nc = (uint32_t)inv[c]; }
    else if (mode == 1) { nr = (uint32_t)c; nc = (uint32_t)r; }
    else { nr = (uint32_t)r; nc = (uint32_t)c; }
    keys[e] = (nr << colbits) | nc;
    ids[e] = (int32_t)e;
  }
}

__global__ void k_flags(const uint64_t* __restrict__ keys, int64_t nnz, int32_t* __restrict__ f) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= nnz; i += stride)
    f[i] = (i < nnz && (i == 0 || keys[i] != keys[i - 1])) ? 1 : 0;
}

// One thread per distinct pair: column, value sum (input CSR order) and row.
__global__ void k_emit(const uint64_t* __restrict__ keys, const int32_t* __restrict__ ids,
                       const int32_t* __restrict__ P, const float* __restrict__ val, int64_t nnz,
                       int colbits, int32_t* __restrict__ col_out, float* __restrict__ val_out,
                       int32_t* __restrict__ row_sorted) {
  const uint64_t cmask = (1ull << colbits) - 1;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += stride) {
    const uint64_t k = keys[i];
    if (i > 0 && keys[i - 1] == k) continue;
    const int32_t o = P[i];
    col_out[o] = (int32_t)(k & cmask);
    row_sorted[o] = (int32_t)(k >> colbits);
    if (val_out) {
      float s = val ? val[ids[i]] : 1.0f;
      for (int64_t j = i + 1; j < nnz && keys[j] == k; ++j) s += val ? val[ids[j]] : 1.0f;
      val_out[o] = s;
    }
  }
}

// rowptr_out[r] = first output position of a row >= r.
__global__ void k_rowptr(const int32_t* __restrict__ row_sorted, int64_t n, int32_t rows,
                         int32_t* __restrict__ rowptr) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += stride) {
    const int32_t prev = (i == 0) ? -1 : row_sorted[i - 1];
    const int32_t cur = (i == n) ? rows : row_sorted[i];
    for (int32_t r = prev + 1; r <= cur; ++r) rowptr[r] = (int32_t)i;
  }
}

struct Layout {
  size_t inv, seen, erow, keys_in, keys_out, ids_in, ids_out, flags, P, rsort, bad, sort, scan;
  size_t total;
  int colbits, endbit;
};

Layout layout(int32_t rows_in, int32_t cols_in, int64_t nnz, int mode) {
  Layout L{};
  const int32_t rows_out = mode == 1 ? cols_in : rows_in;
  const int32_t cols_out = mode == 1 ? rows_in : cols_in;
  L.colbits = bits_for((uint64_t)(cols_out > 0 ? cols_out : 1));
  L.endbit = L.colbits + bits_for((uint64_t)(rows_out > 0 ? rows_out : 1));
  const size_t n = (size_t)(nnz > 0 ? nnz : 1);
  const size_t m = (size_t)(rows_in > 0 ? rows_in : 1);
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + bytes, 256); return o; };
  L.inv = take(m * 4);
  L.seen = take(m * 4);
  L.erow = take(n * 4);
  L.keys_in = take(n * 8);
  L.keys_out = take(n * 8);
  L.ids_in = take(n * 4);
  L.ids_out = take(n * 4);
  L.flags = take((n + 1) * 4);
  L.P = take((n + 1) * 4);
  L.rsort = take(n * 4);
  L.bad = take(16);
  size_t s1 = 0, s2 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, s1, (uint64_t*)nullptr, (uint64_t*)nullptr,
                                  (int32_t*)nullptr, (int32_t*)nullptr, (int64_t)n, 0, L.endbit);
  cub::DeviceScan::ExclusiveSum(nullptr, s2, (int32_t*)nullptr, (int32_t*)nullptr,
                                (int64_t)n + 1);
  L.sort = take(s1);
  L.scan = take(s2);
  L.total = off;
  return L;
}

dtc_status relabel(int mode, const int32_t* rowptr, const int32_t* col, const float* val,
                   int32_t M, int32_t K, int64_t nnz, const int32_t* perm, int32_t* rowptr_out,
                   int32_t* col_out, float* val_out, int64_t* nnz_out, void* ws, size_t wsb,
                   cudaStream_t st) {
  DTC_REQUIRE(M >= 0 && K >= 0 && nnz >= 0, "negative sizes");
  DTC_REQUIRE(M > 0 || nnz == 0, "a matrix without rows has no entries");
  DTC_REQUIRE(nnz < (int64_t)INT32_MAX, "nnz must fit in int32");
  DTC_REQUIRE(nnz_out != nullptr, "nnz_out is null");
  DTC_REQUIRE((rowptr || (mode == 2 && nnz == 0)) && rowptr_out, "null device pointer");
  DTC_REQUIRE(nnz == 0 || (col && col_out), "null device pointer");
  DTC_REQUIRE(mode != 0 || perm || M == 0, "perm is null");
  const Layout L = layout(M, K, nnz, mode);
  if (!ws || wsb < L.total) {
    set_error("relabel workspace too small");
    return DTC_ERR_WORKSPACE_TOO_SMALL;
  }
  char* w = (char*)ws;
  int32_t* inv = (int32_t*)(w + L.inv);
  int32_t* seen = (int32_t*)(w + L.seen);
  int32_t* erow = (int32_t*)(w + L.erow);
  uint64_t* kin = (uint64_t*)(w + L.keys_in);
  uint64_t* kout = (uint64_t*)(w + L.keys_out);
  int32_t* iin = (int32_t*)(w + L.ids_in);
  int32_t* iout = (int32_t*)(w + L.ids_out);
  int32_t* flags = (int32_t*)(w + L.flags);
  int32_t* P = (int32_t*)(w + L.P);
  int32_t* rsort = (int32_t*)(w + L.rsort);
  uint32_t* bad = (uint32_t*)(w + L.bad);
  const int32_t rows_out = mode == 1 ? K : M;
  DTC_CUDA(cudaMemsetAsync(bad, 0, 4, st));
  if (mode == 0 && M > 0) {
    DTC_CUDA(cudaMemsetAsync(seen, 0, (size_t)M * 4, st));
    k_invert<<<grid_for(M), kThreads, 0, st>>>(perm, M, inv, seen, bad);
  }
  if (mode == 2) {
    if (nnz > 0) k_coo_rows<<<grid_for(nnz), kThreads, 0, st>>>(rowptr, col, M, K, nnz, erow, bad);
  } else if (M > 0) {
    k_rows<<<grid_for(nnz > M ? nnz : (int64_t)M), kThreads, 0, st>>>(rowptr, col, M, K, nnz, erow,
                                                                     bad);
  }
  uint32_t hbad = 0;
  DTC_CUDA(cudaMemcpyAsync(&hbad, bad, 4, cudaMemcpyDeviceToHost, st));
  DTC_CUDA(cudaStreamSynchronize(st));
  if (hbad & 1u) {
    set_error("perm is not a permutation of [0, num_nodes)");
    return DTC_ERR_INVALID_ARGUMENT;
  }
  if (hbad & 2u) {
    set_error(mode == 2 ? "invalid COO (a coordinate out of range)"
                        : "invalid CSR (rowptr not monotone from 0 to nnz, or a column out of range)");
    return DTC_ERR_INVALID_ARGUMENT;
  }
  if (nnz == 0) {
    DTC_CUDA(cudaMemsetAsync(rowptr_out, 0, ((size_t)rows_out + 1) * 4, st));
    *nnz_out = 0;
    return DTC_OK;
  }
  k_keys<<<grid_for(nnz), kThreads, 0, st>>>(erow, col, inv, nnz, mode, L.colbits, M, K, kin, iin);
  size_t sb = L.scan - L.sort;
  DTC_CUDA(cub::DeviceRadixSort::SortPairs(w + L.sort, sb, kin, kout, iin, iout, nnz, 0, L.endbit,
                                           st));
  k_flags<<<grid_for(nnz + 1), kThreads, 0, st>>>(kout, nnz, flags);
  size_t cb = L.total - L.scan;
  DTC_CUDA(cub::DeviceScan::ExclusiveSum(w + L.scan, cb, flags, P, nnz + 1, st));
  int32_t hn = 0;
  DTC_CUDA(cudaMemcpyAsync(&hn, P + nnz, 4, cudaMemcpyDeviceToHost, st));
  k_emit<<<grid_for(nnz), kThreads, 0, st>>>(kout, iout, P, val, nnz, L.colbits, col_out, val_out,
                                             rsort);
  DTC_CUDA(cudaStreamSynchronize(st));
  k_rowptr<<<grid_for((int64_t)hn + 1), kThreads, 0, st>>>(rsort, hn, rows_out, rowptr_out);
  DTC_CUDA(cudaGetLastError());
  *nnz_out = hn;
  return DTC_OK;
}

}  // namespace
}  // namespace dtc

using namespace dtc;

extern "C" {

dtc_status dtc_relabel_workspace_bytes(int32_t num_rows, int32_t num_cols, int64_t nnz,
                                       size_t* bytes) {
  DTC_REQUIRE(bytes != nullptr, "bytes is null");
  DTC_REQUIRE(num_rows >= 0 && num_cols >= 0 && nnz >= 0, "negative sizes");
  // modes 0 and 2 share a layout
  const Layout a = layout(num_rows, num_cols, nnz, 0), b = layout(num_rows, num_cols, nnz, 1);
  *bytes = a.total > b.total ? a.total : b.total;
  return DTC_OK;
}

dtc_status dtc_permute_csr(const int32_t* d_rowptr, const int32_t* d_col, const float* d_val,
                           int32_t num_nodes, int64_t nnz, const int32_t* d_perm,
                           int32_t* d_rowptr_out, int32_t* d_col_out, float* d_val_out,
                           int64_t* nnz_out, void* d_workspace, size_t workspace_bytes,
                           dtc_stream_t stream) {
  return relabel(0, d_rowptr, d_col, d_val, num_nodes, num_nodes, nnz, d_perm, d_rowptr_out,
                 d_col_out, d_val_out, nnz_out, d_workspace, workspace_bytes,
                 (cudaStream_t)stream);
}

dtc_status dtc_transpose_csr(const int32_t* d_rowptr, const int32_t* d_col, const float* d_val,
                             int32_t num_rows, int32_t num_cols, int64_t nnz,
                             int32_t* d_rowptr_out, int32_t* d_col_out, float* d_val_out,
                             int64_t* nnz_out, void* d_workspace, size_t workspace_bytes,
                             dtc_stream_t stream) {
  return relabel(1, d_rowptr, d_col, d_val, num_rows, num_cols, nnz, nullptr, d_rowptr_out,
                 d_col_out, d_val_out, nnz_out, d_workspace, workspace_bytes,
                 (cudaStream_t)stream);
}

dtc_status dtc_coo_to_csr(const int32_t* d_src, const int32_t* d_dst, const float* d_val,
                          int32_t num_rows, int32_t num_cols, int64_t nnz, int32_t* d_rowptr_out,
                          int32_t* d_col_out, float* d_val_out, int64_t* nnz_out,
                          void* d_workspace, size_t workspace_bytes, dtc_stream_t stream) {
  return relabel(2, d_src, d_dst, d_val, num_rows, num_cols, nnz, nullptr,
                 d_rowptr_out, d_col_out, d_val_out, nnz_out, d_workspace, workspace_bytes,
                 (cudaStream_t)stream);
}

}  // extern "C"
