// ME-TCF conversion on the GPU, fully parallel (no per-window serial loops).
//
// Output semantics follow the reference conversion bit for bit
// (DTC-SpMM/DTCSpMM_kernel.cu:107-419, DTC-SpMM/DTCSpMM.cpp:313-359):
//   window w = rows [w*H, min(w*H+H, M)); U_w = sorted distinct columns of w;
//   blockPartition[w] = ceil(|U_w|/W) (0 for empty windows);
//   edgeToColumn[e] = rank of col(e) in U_w; block = rank / W, slot = rank % W;
//   TCblocktileId entries of a block are stored in CSR edge order;
//   SparseAToX[b*W + slot] = column (0 in unused slots).
// The reference computes U_w and the per-block scatter with one thread per
// window (:234-240, :309-329); here both steps are radix sorts + scans:
//   phase 1: sort (window, col) keys -> distinct flags -> scan -> ranks;
//   phase 2: stable sort of edges by global block id -> offsets, tile ids.
#include <cub/cub.cuh>
#include "common.cuh"

namespace dtc {
namespace {

constexpr int kThreads = 256;

inline int bits_for(uint64_t n) {  // bits to represent values in [0, n)
  int b = 0;
  while (b < 63 && (1ull << b) < n) ++b;
  return b < 1 ? 1 : b;
}

inline unsigned grid_for(int64_t n, int per = kThreads) {
  int64_t g = (n + per - 1) / per;
  if (g < 1) g = 1;
  if (g > (1 << 30)) g = 1 << 30;
  return (unsigned)g;
}

// Validates CSR structure: rowptr[0] == 0, rowptr non-decreasing,
// rowptr[M] == nnz, 0 <= col < num_cols. Sets bits in *bad.
__global__ void k_validate(const int32_t* __restrict__ col, const int32_t* __restrict__ rowptr,
                           int32_t M, int64_t nnz, int32_t num_cols, uint32_t* bad) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = i; r <= M; r += stride) {
    int32_t v = rowptr[r];
    if (r == 0 && v != 0) atomicOr(bad, 1u);
    if (r == M && v != nnz) atomicOr(bad, 2u);
    if (r < M && rowptr[r + 1] < v) atomicOr(bad, 4u);
  }
  for (int64_t e = i; e < nnz; e += stride) {
    int32_t c = col[e];
    if (c < 0 || c >= num_cols) atomicOr(bad, 8u);
  }
}

// edgeToRow[e] = row (DTCSpMM_kernel.cu:107-120): one warp per row.
__global__ void k_edge_to_row(const int32_t* __restrict__ rowptr, int32_t M,
                              int32_t* __restrict__ edgeToRow) {
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < M; r += nwarps) {
    int32_t e1 = rowptr[r + 1];
    for (int32_t e = rowptr[r] + lane; e < e1; e += 32) edgeToRow[e] = (int32_t)r;
  }
}

// Sort keys (window << colbits | col) and edge ids.
template <typename K>
__global__ void k_make_keys(const int32_t* __restrict__ col, const int32_t* __restrict__ edgeToRow,
                            int64_t nnz, int32_t H, int colbits, K* __restrict__ keys,
                            int32_t* __restrict__ ids) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += stride) {
    K w = (K)(edgeToRow[e] / H);
    keys[e] = (w << colbits) | (K)(uint32_t)col[e];
    ids[e] = (int32_t)e;
  }
}

// flags[i] = 1 where sorted key i starts a new (window, col) pair; flags[nnz] = 0.
template <typename K>
__global__ void k_distinct_flags(const K* __restrict__ keys, int64_t nnz, int32_t* __restrict__ flags) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= nnz; i += stride)
    flags[i] = (i < nnz && (i == 0 || keys[i] != keys[i - 1])) ? 1 : 0;
}

// edgeToColumn[e] = rank of col(e) among the window's distinct columns:
// P = exclusive scan of flags (P[nnz] = #distinct pairs); the window's sorted
// range equals its CSR edge range, so rank(i) = P[i+1] - 1 - P[rowptr[w*H]].
template <typename K>
__global__ void k_ranks(const K* __restrict__ keys, const int32_t* __restrict__ ids,
                        const int32_t* __restrict__ P, const int32_t* __restrict__ rowptr, int64_t nnz,
                        int32_t H, int colbits, int32_t* __restrict__ edgeToColumn) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nnz; i += stride) {
    int32_t w = (int32_t)(keys[i] >> colbits);
    int32_t s = rowptr[(int64_t)w * H];
    edgeToColumn[ids[i]] = P[i + 1] - 1 - P[s];
  }
}

// blockPartition[w] = ceil(U_w / W) (0 for empty windows, :215-227).
__global__ void k_block_partition(const int32_t* __restrict__ P, const int32_t* __restrict__ rowptr,
                                  int32_t M, int32_t nwin, int32_t H, int32_t W,
                                  int32_t* __restrict__ blockPartition, int32_t* __restrict__ bp_ext) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w <= nwin; w += stride) {
    if (w == nwin) { bp_ext[w] = 0; continue; }
    int64_t r1 = w * H + H;
    if (r1 > M) r1 = M;
    int32_t u = P[rowptr[r1]] - P[rowptr[w * H]];
    int32_t nb = (u + W - 1) / W;
    blockPartition[w] = nb;
    bp_ext[w] = nb;
  }
}

// TCblockRowid[b] = w (:149-173); one warp per window.
__global__ void k_block_rowid(const int32_t* __restrict__ rwo, int32_t nwin,
                              int32_t* __restrict__ rowid) {
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t w = warp; w < nwin; w += nwarps) {
    int32_t b1 = rwo[w + 1];
    for (int32_t b = rwo[w] + lane; b < b1; b += 32) rowid[b] = (int32_t)w;
  }
}

// Global block id of each edge (CSR order) for the stable sort.
__global__ void k_edge_block(const int32_t* __restrict__ edgeToColumn,
                             const int32_t* __restrict__ edgeToRow, const int32_t* __restrict__ rwo,
                             int64_t nnz, int32_t H, int32_t W, uint32_t* __restrict__ blk,
                             int32_t* __restrict__ ids) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += stride) {
    blk[e] = (uint32_t)(rwo[edgeToRow[e] / H] + edgeToColumn[e] / W);
    ids[e] = (int32_t)e;
  }
}

// Per sorted position j (edges grouped by block, CSR order inside a block):
// block offsets, tile ids (:287-300) and SparseAToX (:296).
__global__ void k_scatter_tiles(const uint32_t* __restrict__ blk_sorted,
                                const int32_t* __restrict__ ids_sorted,
                                const int32_t* __restrict__ col, const int32_t* __restrict__ edgeToColumn,
                                const int32_t* __restrict__ edgeToRow, int64_t nnz, int64_t T,
                                int32_t H, int32_t W, int32_t* __restrict__ tcblockOffset,
                                uint8_t* __restrict__ tileId, int32_t* __restrict__ sparseAToX) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nnz; j += stride) {
    int32_t b = (int32_t)blk_sorted[j];
    if (j == 0 || (int32_t)blk_sorted[j - 1] != b) {
      // every TC block holds at least one edge, so offsets are run starts
      int32_t prev = (j == 0) ? -1 : (int32_t)blk_sorted[j - 1];
      for (int32_t q = prev + 1; q <= b; ++q) tcblockOffset[q] = (int32_t)j;
    }
    if (j == nnz - 1) tcblockOffset[T] = (int32_t)nnz;
    int32_t e = ids_sorted[j];
    int32_t rk = edgeToColumn[e];
    int32_t slot = rk % W;
    tileId[j] = (uint8_t)((edgeToRow[e] % H) * W + slot);
    sparseAToX[(int64_t)b * W + slot] = col[e];  // duplicates write the same value
  }
}

// Values in tile order; duplicate (row, col) of a block merged into the
// first occurrence in CSR order (fp32 sum in CSR order), later ones 0.
__global__ void k_tile_values(const int32_t* __restrict__ tcblockOffset,
                              const uint8_t* __restrict__ tileId, const int32_t* __restrict__ ids_sorted,
                              const float* __restrict__ values, int64_t T,
                              float* __restrict__ tcValues) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < T; b += stride) {
    uint32_t seen[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    int32_t j0 = tcblockOffset[b], j1 = tcblockOffset[b + 1];
    for (int32_t j = j0; j < j1; ++j) {
      uint32_t p = tileId[j];
      float v = values[ids_sorted[j]];
      uint32_t bit = 1u << (p & 31);
      if (!(seen[p >> 5] & bit)) {
        seen[p >> 5] |= bit;
        tcValues[j] = v;
      } else {
        int32_t f = j0;
        while (tileId[f] != p) ++f;
        tcValues[f] += v;
        tcValues[j] = 0.0f;
      }
    }
  }
}

struct Phase1Layout {
  size_t keys_in, keys_out, ids_in, ids_out, flags, P, bp_ext, bad, cub_sort, cub_scan, total;
  bool wide;
  int colbits, endbit;
};

struct Phase2Layout {
  size_t blk_in, blk_out, ids_in, ids_out, cub_sort, total;
  int endbit;
};

Phase1Layout phase1_layout(int32_t M, int64_t nnz, int32_t H) {
  Phase1Layout L{};
  int32_t nwin = (M + H - 1) / H;
  L.colbits = bits_for((uint64_t)(M > 0 ? M : 1));
  int winbits = bits_for((uint64_t)(nwin > 0 ? nwin : 1));
  L.endbit = L.colbits + winbits;
  L.wide = L.endbit > 32;
  size_t ks = L.wide ? 8 : 4;
  size_t n = (size_t)(nnz > 0 ? nnz : 1);
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + bytes, 256); return o; };
  L.keys_in = take(n * ks);
  L.keys_out = take(n * ks);
  L.ids_in = take(n * 4);
  L.ids_out = take(n * 4);
  L.flags = take((n + 1) * 4);
  L.P = take((n + 1) * 4);
  L.bp_ext = take((size_t)(nwin + 1) * 4);
  L.bad = take(16);
  size_t s1 = 0, s2 = 0, s3 = 0;
  if (L.wide) {
    cub::DeviceRadixSort::SortPairs(nullptr, s1, (uint64_t*)nullptr, (uint64_t*)nullptr,
                                    (int32_t*)nullptr, (int32_t*)nullptr, (int64_t)n, 0, L.endbit);
  } else {
    cub::DeviceRadixSort::SortPairs(nullptr, s1, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (int32_t*)nullptr, (int32_t*)nullptr, (int64_t)n, 0, L.endbit);
  }
  cub::DeviceScan::ExclusiveSum(nullptr, s2, (int32_t*)nullptr, (int32_t*)nullptr, (int64_t)n + 1);
  cub::DeviceScan::ExclusiveSum(nullptr, s3, (int32_t*)nullptr, (int32_t*)nullptr,
                                (int64_t)nwin + 1);
  L.cub_sort = take(s1);
  L.cub_scan = take(s2 > s3 ? s2 : s3);
  L.total = off;
  return L;
}

Phase2Layout phase2_layout(int64_t nnz, int64_t T_upper) {
  Phase2Layout L{};
  size_t n = (size_t)(nnz > 0 ? nnz : 1);
  L.endbit = bits_for((uint64_t)(T_upper > 0 ? T_upper : 1));
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align_up(off + bytes, 256); return o; };
  L.blk_in = take(n * 4);
  L.blk_out = take(n * 4);
  L.ids_in = take(n * 4);
  L.ids_out = take(n * 4);
  size_t s1 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, s1, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (int32_t*)nullptr, (int32_t*)nullptr, (int64_t)n, 0, L.endbit);
  L.cub_sort = take(s1);
  L.total = off;
  return L;
}

template <typename K>
dtc_status phase1_sort(const Phase1Layout& L, char* ws, const int32_t* col, const int32_t* rowptr,
                       int32_t M, int64_t nnz, int32_t H, int32_t* edgeToRow, int32_t* edgeToColumn,
                       cudaStream_t st) {
  K* keys_in = (K*)(ws + L.keys_in);
  K* keys_out = (K*)(ws + L.keys_out);
  int32_t* ids_in = (int32_t*)(ws + L.ids_in);
  int32_t* ids_out = (int32_t*)(ws + L.ids_out);
  int32_t* flags = (int32_t*)(ws + L.flags);
  int32_t* P = (int32_t*)(ws + L.P);
  k_make_keys<K><<<grid_for(nnz), kThreads, 0, st>>>(col, edgeToRow, nnz, H, L.colbits, keys_in,
                                                     ids_in);
  size_t tb = L.cub_scan - L.cub_sort;
  DTC_CUDA(cub::DeviceRadixSort::SortPairs(ws + L.cub_sort, tb, keys_in, keys_out, ids_in, ids_out,
                                           nnz, 0, L.endbit, st));
  k_distinct_flags<K><<<grid_for(nnz + 1), kThreads, 0, st>>>(keys_out, nnz, flags);
  size_t sb = L.total - L.cub_scan;
  DTC_CUDA(cub::DeviceScan::ExclusiveSum(ws + L.cub_scan, sb, flags, P, nnz + 1, st));
  k_ranks<K><<<grid_for(nnz), kThreads, 0, st>>>(keys_out, ids_out, P, rowptr, nnz, H, L.colbits,
                                                 edgeToColumn);
  return DTC_OK;
}

}  // namespace
}  // namespace dtc

using namespace dtc;

extern "C" dtc_status dtc_convert_workspace_bytes(int32_t num_nodes, int64_t nnz, int32_t block_h,
                                                  int32_t block_w, size_t* bytes) {
  DTC_REQUIRE(bytes != nullptr, "bytes is null");
  DTC_REQUIRE(num_nodes >= 0 && nnz >= 0 && block_h > 0 && block_w > 0,
              "negative sizes or non-positive block shape");
  DTC_REQUIRE(block_h * block_w <= 256, "block_h * block_w must be <= 256 (u8 tile ids)");
  DTC_REQUIRE(nnz < (int64_t)INT32_MAX, "nnz must fit in int32 (reference index type)");
  Phase1Layout a = phase1_layout(num_nodes, nnz, block_h);
  Phase2Layout b = phase2_layout(nnz, nnz);
  *bytes = a.total > b.total ? a.total : b.total;
  return DTC_OK;
}

extern "C" dtc_status dtc_convert_count(const int32_t* d_col, const int32_t* d_rowptr,
                                        int32_t num_nodes, int64_t nnz, int32_t block_h,
                                        int32_t block_w, int32_t* d_blockPartition,
                                        int32_t* d_edgeToColumn, int32_t* d_edgeToRow,
                                        int32_t* d_rowWindowOffset, void* d_workspace,
                                        size_t workspace_bytes, int64_t* num_blocks,
                                        dtc_stream_t stream) {
  size_t need = 0;
  dtc_status s = dtc_convert_workspace_bytes(num_nodes, nnz, block_h, block_w, &need);
  if (s != DTC_OK) return s;
  DTC_REQUIRE(num_blocks != nullptr, "num_blocks is null");
  DTC_REQUIRE(d_rowptr && d_blockPartition && d_rowWindowOffset, "null device pointer");
  DTC_REQUIRE(nnz == 0 || (d_col && d_edgeToColumn && d_edgeToRow), "null device pointer");
  if (workspace_bytes < need || d_workspace == nullptr) {
    set_error("conversion workspace too small");
    return DTC_ERR_WORKSPACE_TOO_SMALL;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int32_t nwin = (num_nodes + block_h - 1) / block_h;
  Phase1Layout L = phase1_layout(num_nodes, nnz, block_h);
  char* ws = (char*)d_workspace;
  uint32_t* bad = (uint32_t*)(ws + L.bad);
  DTC_CUDA(cudaMemsetAsync(bad, 0, 4, st));
  k_validate<<<grid_for((nnz > num_nodes ? nnz : num_nodes) + 1), kThreads, 0, st>>>(
      d_col, d_rowptr, num_nodes, nnz, num_nodes, bad);
  if (nnz > 0) {
    k_edge_to_row<<<grid_for((int64_t)num_nodes * 32), kThreads, 0, st>>>(d_rowptr, num_nodes,
                                                                           d_edgeToRow);
    s = L.wide ? phase1_sort<uint64_t>(L, ws, d_col, d_rowptr, num_nodes, nnz, block_h, d_edgeToRow,
                                       d_edgeToColumn, st)
               : phase1_sort<uint32_t>(L, ws, d_col, d_rowptr, num_nodes, nnz, block_h, d_edgeToRow,
                                       d_edgeToColumn, st);
    if (s != DTC_OK) return s;
  } else {
    DTC_CUDA(cudaMemsetAsync(ws + L.P, 0, 4, st));
  }
  int32_t* bp_ext = (int32_t*)(ws + L.bp_ext);
  if (nwin > 0) {
    k_block_partition<<<grid_for((int64_t)nwin + 1), kThreads, 0, st>>>(
        (int32_t*)(ws + L.P), d_rowptr, num_nodes, nwin, block_h, block_w, d_blockPartition,
        bp_ext);
    size_t sb = L.total - L.cub_scan;
    DTC_CUDA(cub::DeviceScan::ExclusiveSum(ws + L.cub_scan, sb, bp_ext, d_rowWindowOffset,
                                           (int64_t)nwin + 1, st));
  } else {
    DTC_CUDA(cudaMemsetAsync(d_rowWindowOffset, 0, 4, st));
  }
  int32_t hostv[2] = {0, 0};
  DTC_CUDA(cudaMemcpyAsync(&hostv[0], d_rowWindowOffset + nwin, 4, cudaMemcpyDeviceToHost, st));
  DTC_CUDA(cudaMemcpyAsync(&hostv[1], bad, 4, cudaMemcpyDeviceToHost, st));
  DTC_CUDA(cudaStreamSynchronize(st));
  if (hostv[1] != 0) {
    set_error("invalid CSR input (flags " + std::to_string(hostv[1]) +
              "): need rowptr[0]==0, non-decreasing rowptr, rowptr[M]==nnz, 0<=col<M");
    return DTC_ERR_INVALID_ARGUMENT;
  }
  *num_blocks = hostv[0];
  return DTC_OK;
}

extern "C" dtc_status dtc_convert_fill(const int32_t* d_col, const int32_t* d_rowptr,
                                       int32_t num_nodes, int64_t nnz, int32_t block_h,
                                       int32_t block_w, const int32_t* d_edgeToColumn,
                                       const int32_t* d_edgeToRow,
                                       const int32_t* d_rowWindowOffset, int64_t num_blocks,
                                       int32_t* d_tcblockRowid, uint8_t* d_tileId,
                                       int32_t* d_tcblockOffset, int32_t* d_sparseAToX,
                                       const float* d_values, float* d_tcValues,
                                       void* d_workspace, size_t workspace_bytes,
                                       dtc_stream_t stream) {
  size_t need = 0;
  dtc_status s = dtc_convert_workspace_bytes(num_nodes, nnz, block_h, block_w, &need);
  if (s != DTC_OK) return s;
  DTC_REQUIRE(num_blocks >= 0 && num_blocks <= nnz, "num_blocks out of range");
  DTC_REQUIRE(d_tcblockOffset != nullptr, "null tcblockOffset");
  DTC_REQUIRE((d_values == nullptr) == (d_tcValues == nullptr),
              "values and tcValues must both be set or both be null");
  if (workspace_bytes < need || d_workspace == nullptr) {
    set_error("conversion workspace too small");
    return DTC_ERR_WORKSPACE_TOO_SMALL;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int32_t nwin = (num_nodes + block_h - 1) / block_h;
  if (num_blocks == 0 || nnz == 0) {
    DTC_CUDA(cudaMemsetAsync(d_tcblockOffset, 0, 4, st));
    return DTC_OK;
  }
  Phase2Layout L = phase2_layout(nnz, num_blocks);
  char* ws = (char*)d_workspace;
  uint32_t* blk_in = (uint32_t*)(ws + L.blk_in);
  uint32_t* blk_out = (uint32_t*)(ws + L.blk_out);
  int32_t* ids_in = (int32_t*)(ws + L.ids_in);
  int32_t* ids_out = (int32_t*)(ws + L.ids_out);
  k_block_rowid<<<grid_for((int64_t)nwin * 32), kThreads, 0, st>>>(d_rowWindowOffset, nwin,
                                                                   d_tcblockRowid);
  DTC_CUDA(cudaMemsetAsync(d_sparseAToX, 0, (size_t)num_blocks * block_w * 4, st));
  k_edge_block<<<grid_for(nnz), kThreads, 0, st>>>(d_edgeToColumn, d_edgeToRow, d_rowWindowOffset,
                                                   nnz, block_h, block_w, blk_in, ids_in);
  size_t tb = L.total - L.cub_sort;
  DTC_CUDA(cub::DeviceRadixSort::SortPairs(ws + L.cub_sort, tb, blk_in, blk_out, ids_in, ids_out,
                                           nnz, 0, L.endbit, st));
  k_scatter_tiles<<<grid_for(nnz), kThreads, 0, st>>>(blk_out, ids_out, d_col, d_edgeToColumn,
                                                      d_edgeToRow, nnz, num_blocks, block_h,
                                                      block_w, d_tcblockOffset, d_tileId,
                                                      d_sparseAToX);
  if (d_values) {
    k_tile_values<<<grid_for(num_blocks), kThreads, 0, st>>>(d_tcblockOffset, d_tileId, ids_out,
                                                             d_values, num_blocks, d_tcValues);
  }
  DTC_CUDA(cudaGetLastError());
  return DTC_OK;
}
