// 48-dimensional structural feature vector of a sparse matrix and its ME-TCF
// form: the input of the learned schedule cost model.
//
//   [ 0,16) row-length histogram: bin 0 = empty rows, bin 1+j = lengths in
//           [2^j, 2^(j+1)), last bin open-ended; fractions of rows
//   [16,28) TC blocks per row window, same binning (bin 0 = empty windows)
//   [28,36) nonzeros per TC block: bins [1], [2,4), [4,8), ... [64,128), [128]
//   36 log2(rows)/24         37 log2(nnz)/28        38 log2(T)/26
//   39 log2(N)/10            40 log2(nnz/rows)/10   41 log2(max row length)/16
//   42 U/nnz: gathered B rows per nonzero (U = distinct (window, column) pairs)
//   43 8T/U: padding of the last block of each window (>= 1)
//   44 mean |col - row| / rows          45 fraction of nonzeros with |col - row| < 64
//   46 coefficient of variation of blocks per window / 10
//   47 fraction of windows without nonzeros
// All accumulation is in 64-bit integers (order independent), so the vector is
// bitwise reproducible and equal to a CPU recomputation that finishes in double
// and rounds to float.
#include "common.cuh"

namespace dtc {
namespace {

constexpr int kThreads = 256;
enum : int {  // integer accumulator slots
  kRowHist = 0,      // 16
  kWinHist = 16,     // 12
  kBlkHist = 28,     // 8
  kMaxLen = 36,
  kU = 37,
  kAbsDist = 38,
  kNear = 39,
  kSumBp2 = 40,
  kSlots = 41,
};

__device__ __forceinline__ int log_bin(int64_t v, int nbins) {  // v >= 1
  int b = 63 - __clzll((unsigned long long)v);                  // floor(log2 v)
  b += 1;
  return b < nbins - 1 ? b : nbins - 1;
}

__global__ void k_row_stats(const int32_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                            int32_t M, unsigned long long* acc) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < M; r += nwarps) {
    const int32_t e0 = rowptr[r], e1 = rowptr[r + 1];
    const int64_t len = e1 - e0;
    unsigned long long dist = 0, near = 0;
    for (int32_t e = e0 + lane; e < e1; e += 32) {
      const int64_t d = (int64_t)col[e] - r;
      const int64_t a = d < 0 ? -d : d;
      dist += (unsigned long long)a;
      near += a < 64 ? 1ull : 0ull;
    }
    for (int o = 16; o; o >>= 1) {
      dist += __shfl_xor_sync(0xffffffffu, dist, o);
      near += __shfl_xor_sync(0xffffffffu, near, o);
    }
    if (lane == 0) {
      atomicAdd(acc + kRowHist + (len == 0 ? 0 : log_bin(len, 16)), 1ull);
      atomicMax(acc + kMaxLen, (unsigned long long)len);
      atomicAdd(acc + kAbsDist, dist);
      atomicAdd(acc + kNear, near);
    }
  }
}

// Per window: blocks (rwo), distinct columns U_w = 1 + max rank (edgeToColumn).
__global__ void k_window_stats(const int32_t* __restrict__ rowptr,
                               const int32_t* __restrict__ rwo,
                               const int32_t* __restrict__ e2c, int32_t M, int32_t nwin,
                               unsigned long long* acc) {
  const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t w = warp; w < nwin; w += nwarps) {
    const int64_t bp = rwo[w + 1] - rwo[w];
    const int64_t r0 = w * 16, r1 = (w * 16 + 16 < M) ? w * 16 + 16 : M;
    const int32_t e0 = rowptr[r0], e1 = rowptr[r1];
    int32_t mx = -1;
    for (int32_t e = e0 + lane; e < e1; e += 32) mx = max(mx, e2c[e]);
    for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) {
      atomicAdd(acc + kWinHist + (bp == 0 ? 0 : log_bin(bp, 12)), 1ull);
      atomicAdd(acc + kU, (unsigned long long)(mx + 1));
      atomicAdd(acc + kSumBp2, (unsigned long long)(bp * bp));
    }
  }
}

__global__ void k_block_stats(const int32_t* __restrict__ toff, int64_t T,
                              unsigned long long* acc) {
  __shared__ unsigned long long h[8];
  if (threadIdx.x < 8) h[threadIdx.x] = 0;
  __syncthreads();
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < T; b += stride) {
    const int64_t n = toff[b + 1] - toff[b];
    int bin = n <= 1 ? 0 : (63 - __clzll((unsigned long long)n));  // [2,4) -> 1 ... [128] -> 7
    bin = bin < 7 ? bin : 7;
    atomicAdd(&h[bin], 1ull);
  }
  __syncthreads();
  if (threadIdx.x < 8 && h[threadIdx.x]) atomicAdd(acc + kBlkHist + threadIdx.x, h[threadIdx.x]);
}

__global__ void k_finish(const unsigned long long* __restrict__ acc, int32_t M, int64_t nnz,
                         int32_t nwin, int64_t T, int32_t N, float* __restrict__ f) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double m = M > 0 ? (double)M : 1.0, w = nwin > 0 ? (double)nwin : 1.0;
  const double t = T > 0 ? (double)T : 1.0, z = nnz > 0 ? (double)nnz : 1.0;
  for (int i = 0; i < 16; ++i) f[i] = (float)((double)acc[kRowHist + i] / m);
  for (int i = 0; i < 12; ++i) f[16 + i] = (float)((double)acc[kWinHist + i] / w);
  for (int i = 0; i < 8; ++i) f[28 + i] = (float)((double)acc[kBlkHist + i] / t);
  const double U = (double)acc[kU];
  f[36] = (float)(log2(m) / 24.0);
  f[37] = (float)(log2(z) / 28.0);
  f[38] = (float)(log2(t) / 26.0);
  f[39] = (float)(log2((double)(N > 0 ? N : 1)) / 10.0);
  f[40] = (float)(log2(z / m) / 10.0);
  f[41] = (float)(log2((double)(acc[kMaxLen] > 0 ? acc[kMaxLen] : 1)) / 16.0);
  f[42] = (float)(U / z);
  f[43] = (float)(U > 0 ? 8.0 * (double)T / U : 1.0);
  f[44] = (float)((double)acc[kAbsDist] / z / m);
  f[45] = (float)((double)acc[kNear] / z);
  const double mean = (double)T / w;
  const double var = (double)acc[kSumBp2] / w - mean * mean;
  f[46] = (float)(mean > 0 ? sqrt(var > 0 ? var : 0.0) / mean / 10.0 : 0.0);
  f[47] = (float)((double)acc[kWinHist + 0] / w);
}

}  // namespace
}  // namespace dtc

using namespace dtc;

extern "C" {

size_t dtc_features_workspace_bytes(void) { return kSlots * sizeof(unsigned long long); }

dtc_status dtc_features(const int32_t* d_rowptr, const int32_t* d_col, int32_t num_nodes,
                        int64_t nnz, const int32_t* d_rowWindowOffset,
                        const int32_t* d_tcblockOffset, const int32_t* d_edgeToColumn,
                        int32_t num_windows, int64_t num_blocks, int32_t N, float* d_features,
                        void* d_workspace, size_t workspace_bytes, dtc_stream_t stream) {
  DTC_REQUIRE(num_nodes >= 0 && nnz >= 0 && num_blocks >= 0 && N >= 1, "bad sizes");
  DTC_REQUIRE(num_windows == (num_nodes + 15) / 16, "num_windows must be ceil(num_nodes/16)");
  DTC_REQUIRE(d_rowptr && d_rowWindowOffset && d_tcblockOffset && d_features, "null pointer");
  DTC_REQUIRE(nnz == 0 || (d_col && d_edgeToColumn), "null pointer");
  if (!d_workspace || workspace_bytes < dtc_features_workspace_bytes()) {
    set_error("features workspace too small");
    return DTC_ERR_WORKSPACE_TOO_SMALL;
  }
  cudaStream_t st = (cudaStream_t)stream;
  auto* acc = (unsigned long long*)d_workspace;
  DTC_CUDA(cudaMemsetAsync(acc, 0, dtc_features_workspace_bytes(), st));
  const int sms = num_sms();
  if (num_nodes > 0)
    k_row_stats<<<sms * 8, kThreads, 0, st>>>(d_rowptr, d_col, num_nodes, acc);
  if (num_windows > 0)
    k_window_stats<<<sms * 8, kThreads, 0, st>>>(d_rowptr, d_rowWindowOffset, d_edgeToColumn,
                                                 num_nodes, num_windows, acc);
  if (num_blocks > 0) k_block_stats<<<sms * 4, kThreads, 0, st>>>(d_tcblockOffset, num_blocks, acc);
  k_finish<<<1, 32, 0, st>>>(acc, num_nodes, nnz, num_windows, num_blocks, N, d_features);
  DTC_CUDA(cudaGetLastError());
  return DTC_OK;
}

}  // extern "C"
