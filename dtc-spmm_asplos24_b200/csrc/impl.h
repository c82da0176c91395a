// Internal entry points shared between the library's translation units (not
// part of the C ABI).
#pragma once
#include "common.cuh"

namespace dtc {

// Epilogue applied to every C element the SpMM writes: C = act(A*B + bias[col]),
// act = ReLU when relu != 0 (the GCN layer's bias + activation).
struct Epilogue {
  const float* bias = nullptr;  // [N] or null
  int relu = 0;
};

dtc_status spmm_tf32_impl(const int32_t* rwo, const uint8_t* tile, const int32_t* toff,
                          const int32_t* s2x, const float* vals, int32_t M, int32_t nwin,
                          int64_t T, const float* B, int32_t N, float* C, int mode, int grid,
                          float* part, cudaStream_t st, int ntile = 0, Epilogue epi = {},
                          int H = 16, void* queue = nullptr, int W = 8);
dtc_status spmm_split_impl(const int32_t* rwo, const uint8_t* tile, const int32_t* toff,
                           const int32_t* s2x, const float* vals, int32_t M, int32_t nwin,
                           int64_t T, int bformat, const void* p0, const void* p1, int32_t N,
                           int precision, float* C, int mode, int grid, float* part,
                           cudaStream_t st, int ntile = 0, Epilogue epi = {}, int H = 16,
                           void* queue = nullptr, int W = 8);
// `queue`: the optional chunk-queue region of a workspace (spmm_queue_bytes,
// 256-byte aligned). With it the kernels run persistent CTAs that pull chunks
// from a counter; without it, one CTA per chunk.
// Tensor map of the row-major fp32 matrix C [M x N] with boxes of 32 columns x
// `box_rows` rows, for TMA stores of finished row-window tiles. Needs C
// 16-byte aligned and N % 4 == 0.
dtc_status encode_c_map(CUtensorMap* map, float* C, int64_t M, int32_t N, int box_rows);
size_t spmm_partials_bytes(int64_t T, int32_t N, int grid, int H = 16);
size_t spmm_queue_bytes(int64_t T, int grid);
dtc_status rowid_to_rwo(const int32_t* rowid, int64_t T, int32_t nwin, int32_t* rwo,
                        cudaStream_t st);
dtc_status spmm_mma_sync_impl(const int32_t* rwo, const uint8_t* tile, const int32_t* toff,
                              const int32_t* s2x, const float* vals, int32_t M, int32_t nwin,
                              const float* B, int32_t N, float* C, cudaStream_t st);
dtc_status pack_b_impl(int fmt, const float* B, int64_t rows, int32_t N, void* p0, void* p1,
                       cudaStream_t st);
dtc_status bformat_bytes_impl(int fmt, int64_t rows, int32_t N, size_t* b0, size_t* b1);

}  // namespace dtc
