// Legacy-ISA TC-block SpMM: mma.sync.m16n8k8 TF32 with B gathered straight
// into registers, one CTA per row window -- the instruction family and
// schedule of the reference kernels (DTC-SpMM/DTCSpMM_kernel.cu:2663-2866),
// written for any N >= 1 with full bounds checks. Used for shapes the TMA
// path cannot take (N % 4 != 0) and as the recompiled-legacy comparison point.
#include "common.cuh"

namespace dtc {
namespace {

constexpr int kWarps = 4;
constexpr int kGroupsPerWarp = 8;                 // n8 feature groups per warp per pass
constexpr int kPassCols = kWarps * kGroupsPerWarp * 8;  // 256 features per pass

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__global__ void __launch_bounds__(kWarps * 32)
    k_spmm_mma_sync(const int32_t* __restrict__ rwo, const uint8_t* __restrict__ tile,
                    const int32_t* __restrict__ toff, const int32_t* __restrict__ s2x,
                    const float* __restrict__ vals, int32_t M, const float* __restrict__ B,
                    int32_t N, float* __restrict__ C, uint32_t* err) {
  __shared__ float a_tile[16 * 8];
  __shared__ int32_t rows[8];
  const int w = blockIdx.x;
  const int pass = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t row0 = (int64_t)w * 16;
  const int32_t b_lo = rwo[w], b_hi = rwo[w + 1];
  const int colbase = pass * kPassCols + warp * kGroupsPerWarp * 8;
  float d[kGroupsPerWarp][4];
#pragma unroll
  for (int g = 0; g < kGroupsPerWarp; ++g) d[g][0] = d[g][1] = d[g][2] = d[g][3] = 0.f;

  for (int32_t b = b_lo; b < b_hi; ++b) {
    a_tile[threadIdx.x] = 0.f;  // 128 threads == 16 x 8 tile
    if (threadIdx.x < 8) {
      int32_t r = s2x[(int64_t)b * 8 + threadIdx.x];
      rows[threadIdx.x] = (threadIdx.x > 0 && r == 0) ? -1 : r;  // padded slot
    }
    __syncthreads();
    for (int32_t e = toff[b] + threadIdx.x; e < toff[b + 1]; e += blockDim.x) {
      uint32_t pos = tile[e];
      float v = vals ? vals[e] : 1.0f;
      if (pos >= 128) { atomicOr(err, kErrBadIndex); continue; }
      if (v != 0.f) a_tile[pos] = v;
    }
    __syncthreads();
    const int gr = lane >> 2, gc = lane & 3;
    uint32_t a0 = to_tf32(a_tile[gr * 8 + gc]);
    uint32_t a1 = to_tf32(a_tile[(gr + 8) * 8 + gc]);
    uint32_t a2 = to_tf32(a_tile[gr * 8 + gc + 4]);
    uint32_t a3 = to_tf32(a_tile[(gr + 8) * 8 + gc + 4]);
    const int32_t rk0 = rows[gc], rk1 = rows[gc + 4];
#pragma unroll
    for (int g = 0; g < kGroupsPerWarp; ++g) {
      const int n = colbase + g * 8 + gr;
      float x0 = 0.f, x1 = 0.f;
      if (n < N) {
        if (rk0 >= 0) x0 = __ldg(B + (int64_t)rk0 * N + n);
        if (rk1 >= 0) x1 = __ldg(B + (int64_t)rk1 * N + n);
      }
      uint32_t b0 = to_tf32(x0), b1 = to_tf32(x1);
      asm volatile(
          "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
          "{%8,%9}, {%0,%1,%2,%3};"
          : "+f"(d[g][0]), "+f"(d[g][1]), "+f"(d[g][2]), "+f"(d[g][3])
          : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    }
    __syncthreads();
  }
  const int gr = lane >> 2, gc = lane & 3;
#pragma unroll
  for (int g = 0; g < kGroupsPerWarp; ++g) {
    const int n0 = colbase + g * 8 + 2 * gc;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t row = row0 + gr + 8 * h;
      if (row >= M) continue;
      if (n0 < N) C[row * N + n0] = d[g][2 * h];
      if (n0 + 1 < N) C[row * N + n0 + 1] = d[g][2 * h + 1];
    }
  }
}

}  // namespace

dtc_status spmm_mma_sync_impl(const int32_t* rwo, const uint8_t* tile, const int32_t* toff,
                              const int32_t* s2x, const float* vals, int32_t M, int32_t nwin,
                              const float* B, int32_t N, float* C, cudaStream_t st) {
  DTC_REQUIRE(M >= 0 && N >= 1, "bad sizes");
  DTC_REQUIRE(nwin == (M + 15) / 16, "num_windows must be ceil(num_nodes/16)");
  if (M == 0) return DTC_OK;
  dim3 grid((unsigned)nwin, (unsigned)((N + kPassCols - 1) / kPassCols));
  k_spmm_mma_sync<<<grid, kWarps * 32, 0, st>>>(rwo, tile, toff, s2x, vals, M, B, N, C,
                                                device_error_word());
  DTC_CUDA(cudaGetLastError());
  return DTC_OK;
}

}  // namespace dtc
