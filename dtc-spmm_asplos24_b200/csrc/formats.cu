// Dense-operand storage forms ("B formats"), produced once and reused by
// every SpMM over the same B:
//   SPLIT24 : fp32 rounded to nearest-even at 16 significant bits and stored
//             as a bf16 "hi" plane plus a u8 "extension" plane (the next 8
//             mantissa bits). 3 bytes/element. In-kernel, lo = b24 - hi is
//             exact in bf16, so (hi, lo) reproduces b24 exactly.
//   BF16    : round-to-nearest-even bf16, 2 bytes/element.
//   FP8     : e4m3 (satfinite, RNE) of B[r,:] / s_r with s_r = max|B[r,:]|/448,
//             plus the fp32 per-row scale s_r. 1 byte/element + 4 bytes/row.
//   BF16X2  : hi = bf16_rn(b), lo = bf16_rn(b - hi) (b - hi is exact in fp32;
//             lo = 0 where hi is not finite), two bf16 planes: 4 bytes/element,
//             hi + lo carries ~16 significant bits and needs no rebuild.
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include "common.cuh"

namespace dtc {
namespace {

__device__ __forceinline__ uint32_t round_to_b24(uint32_t u) {
  const uint32_t e = (u >> 23) & 0xFF;
  if (e == 0xFF) return (u & 0x7FFFFF) ? 0x7FC00000u : u;  // NaN -> canonical, Inf kept
  uint32_t r = u + 0x7Fu + ((u >> 8) & 1u);                // RNE at bit 8
  return r & 0xFFFFFF00u;
}

__global__ void k_pack_split24(const float* __restrict__ B, int64_t n, uint16_t* __restrict__ hi,
                               uint8_t* __restrict__ ext) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    uint32_t r = round_to_b24(__float_as_uint(B[i]));
    hi[i] = (uint16_t)(r >> 16);
    ext[i] = (uint8_t)(r >> 8);
  }
}

__global__ void k_pack_bf16(const float* __restrict__ B, int64_t n, __nv_bfloat16* __restrict__ o) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride)
    o[i] = __float2bfloat16_rn(B[i]);
}

__global__ void k_pack_bf16x2(const float* __restrict__ B, int64_t n, __nv_bfloat16* __restrict__ hi,
                              __nv_bfloat16* __restrict__ lo) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const float b = B[i];
    const __nv_bfloat16 h = __float2bfloat16_rn(b);
    const float hf = __bfloat162float(h);
    hi[i] = h;
    lo[i] = __float2bfloat16_rn(isfinite(hf) ? b - hf : 0.0f);
  }
}

// One warp per row: scale = max|x| / 448, q = e4m3(x / scale).
__global__ void k_pack_fp8(const float* __restrict__ B, int64_t rows, int32_t N,
                           uint8_t* __restrict__ q, float* __restrict__ scale) {
  int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t r = warp; r < rows; r += nw) {
    const float* x = B + r * N;
    float m = 0.f;
    for (int j = lane; j < N; j += 32) m = fmaxf(m, fabsf(x[j]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    const float s = (m > 0.f && isfinite(m)) ? m / 448.0f : 1.0f;
    if (lane == 0) scale[r] = s;
    for (int j = lane; j < N; j += 32)
      q[r * N + j] = (uint8_t)__nv_cvt_float_to_fp8(x[j] / s, __NV_SATFINITE, __NV_E4M3);
  }
}

inline unsigned grid_for(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 64) g = 148 * 64;
  return (unsigned)g;
}

}  // namespace

dtc_status bformat_bytes_impl(int fmt, int64_t rows, int32_t N, size_t* b0, size_t* b1) {
  DTC_REQUIRE(b0 && b1, "null size pointer");
  DTC_REQUIRE(rows >= 0 && N >= 1, "bad sizes");
  size_t n = (size_t)rows * N;
  switch (fmt) {
    case DTC_B_F32: *b0 = n * 4; *b1 = 0; return DTC_OK;
    case DTC_B_SPLIT24: *b0 = n * 2; *b1 = n; return DTC_OK;
    case DTC_B_BF16: *b0 = n * 2; *b1 = 0; return DTC_OK;
    case DTC_B_FP8: *b0 = n; *b1 = (size_t)rows * 4; return DTC_OK;
    case DTC_B_BF16X2: *b0 = n * 2; *b1 = n * 2; return DTC_OK;
  }
  set_error("unknown B format");
  return DTC_ERR_INVALID_ARGUMENT;
}

dtc_status pack_b_impl(int fmt, const float* B, int64_t rows, int32_t N, void* p0, void* p1,
                       cudaStream_t st) {
  DTC_REQUIRE(B && p0, "null device pointer");
  DTC_REQUIRE(rows >= 0 && N >= 1, "bad sizes");
  int64_t n = rows * (int64_t)N;
  if (n == 0) return DTC_OK;
  switch (fmt) {
    case DTC_B_F32:
      DTC_CUDA(cudaMemcpyAsync(p0, B, (size_t)n * 4, cudaMemcpyDeviceToDevice, st));
      return DTC_OK;
    case DTC_B_SPLIT24:
      DTC_REQUIRE(p1, "SPLIT24 needs two planes");
      k_pack_split24<<<grid_for(n), 256, 0, st>>>(B, n, (uint16_t*)p0, (uint8_t*)p1);
      break;
    case DTC_B_BF16:
      k_pack_bf16<<<grid_for(n), 256, 0, st>>>(B, n, (__nv_bfloat16*)p0);
      break;
    case DTC_B_BF16X2:
      DTC_REQUIRE(p1, "BF16X2 needs two planes");
      k_pack_bf16x2<<<grid_for(n), 256, 0, st>>>(B, n, (__nv_bfloat16*)p0, (__nv_bfloat16*)p1);
      break;
    case DTC_B_FP8:
      DTC_REQUIRE(p1, "FP8 needs the scale plane");
      k_pack_fp8<<<grid_for(rows * 32), 256, 0, st>>>(B, rows, N, (uint8_t*)p0, (float*)p1);
      break;
    default:
      set_error("unknown B format");
      return DTC_ERR_INVALID_ARGUMENT;
  }
  DTC_CUDA(cudaGetLastError());
  return DTC_OK;
}

}  // namespace dtc
