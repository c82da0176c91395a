// Issue and completion rate of tcgen05.mma kind::tf32 with M = 128, K = 8 and
// N = 32 (the TF32 SpMM kernel's one instruction per TC block at window height
// 32), 64 and 128 (how the rate scales with the instruction's width), from 1, 2
// or 4 issuing threads of one CTA.
//
// One CTA, zero-filled operand tiles in its own shared memory (32 A tiles in
// the kernel's layout-type-1 swizzle, 4 B tiles), accumulators in TMEM
// (allocated and freed by warp 0), every wait bounded (2 s). Each issuing
// thread issues 4096 back-to-back MMAs over distinct A tiles, commits, and
// waits; the program prints cycles per MMA per thread and for the SM.
//
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -std=c++17 -Iinclude \
//        -Idtc-spmm_asplos24_b200/csrc dtc-spmm_asplos24_b200/microbench/mma_rate.cu -o mma_rate
//   ./mma_rate
#include <cstdio>
#include "common.cuh"
using namespace dtc;

__global__ void __launch_bounds__(128, 1) k_mmabench(int n, int mode, unsigned long long* out,
                                                     uint32_t* err, int nissue, int NN) {
  extern __shared__ uint8_t raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)raw + 1023) & ~(uintptr_t)1023);
  uint8_t* xa = smem;              // 32 A tiles x 4096 B (128 features x 8 rows fp32)
  uint8_t* yb = smem + 32 * 4096;  // 32 B tiles x 1024 B (8 x 32 fp32)
  __shared__ uint64_t bars[8];
  __shared__ uint32_t tslot;
  for (int i = threadIdx.x; i < (32 * 4096 + 32 * 1024) / 16; i += blockDim.x)
    reinterpret_cast<float4*>(smem)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
  fence_proxy_async_smem();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int i = 0; i < 8; ++i) mbar_init(&bars[i], 1);
    fence_mbar_init();
  }
  if (warp == 0) {
    tmem_alloc(&tslot, 512);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tb = tslot;
  const int issuers = nissue;
  const bool same = (mode & 2) != 0;            // bit 1: the same tiles for every MMA
  const bool staged = (mode & 4) != 0;          // bit 2: per 4 MMAs: fences + a commit
  if (warp < issuers && lane == 0) {
    const uint32_t idesc = umma_idesc(2, 128, (uint32_t)NN, 1, 0);
    const uint64_t a0 = umma_desc(smem_u32(xa), 1024, 512, 1);
    const uint64_t b0 = umma_desc(smem_u32(yb), 128, 256, 0);
    const uint32_t d = tb + (uint32_t)(warp * 128);  // up to 128 columns per issuer
    const long long t0 = clock64();
    for (int i = 0; i < n; ++i) {
      if (staged && (i & 3) == 0) {
        fence_proxy_async_smem();
        tc_fence_after();
      }
      const int t = same ? 0 : (i & 31);
      mma_tf32(d, a0 + (uint64_t)((t * 4096) >> 4), b0 + (uint64_t)(((t & 3) * NN * 32) >> 4), idesc,
               i > 0 ? 1u : 0u);
      if (staged && (i & 3) == 3) tc_commit(&bars[4 + warp]);  // never waited: arrivals only
    }
    const long long t1 = clock64();
    tc_commit(&bars[warp]);
    mbar_wait(&bars[warp], 0, err);
    const long long t2 = clock64();
    out[warp * 2 + 0] = (unsigned long long)(t1 - t0);
    out[warp * 2 + 1] = (unsigned long long)(t2 - t0);
  }
  __syncwarp();
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tb, 512);
  }
}

namespace dtc {
void set_error(const std::string&) {}  // the library's error sink, unused here
}

int main() {
  const int smem = 32 * 4096 + 32 * 1024 + 1024;
  cudaFuncSetAttribute(k_mmabench, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  unsigned long long* d_out; uint32_t* d_err;
  cudaMalloc(&d_out, 8 * sizeof(unsigned long long));
  cudaMalloc(&d_err, 4);
  cudaMemset(d_err, 0, 4);
  const int Ns[] = {32, 64, 128, 256};
  const int Is[] = {1, 2, 4};
  for (int r = 0; r < 2; ++r)
    for (int NN : Ns)
      for (int I : Is) {
        if (NN == 256 && I > 2) continue;   // 128 TMEM columns per issuer
        if (NN == 256) continue;            // (N = 256 needs 256 columns per issuer: skipped)
        const int n = 4096;
        cudaMemset(d_out, 0, 8 * sizeof(unsigned long long));
        k_mmabench<<<1, 128, smem>>>(n, 0, d_out, d_err, I, NN);
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) { printf("cuda error %s\n", cudaGetErrorString(e)); return 1; }
        unsigned long long h[8]; uint32_t herr;
        cudaMemcpy(h, d_out, sizeof(h), cudaMemcpyDeviceToHost);
        cudaMemcpy(&herr, d_err, 4, cudaMemcpyDeviceToHost);
        if (r == 1)
          printf("tf32 M128 N%-3d K8, %d issuer(s): per thread issue %.1f complete %.1f cyc/MMA; SM rate %.1f cyc/MMA; err %u\n",
                 NN, I, (double)h[0] / n, (double)h[1] / n, (double)h[1] / n / I, herr);
      }
  // N = 32, one issuer: the same tiles for every MMA (mode 2), and the
  // kernel's per-stage fences and commit every 4 MMAs (mode 4)
  for (int r = 0; r < 2; ++r)
    for (int mode : {2, 4}) {
      const int n = 4096;
      cudaMemset(d_out, 0, 8 * sizeof(unsigned long long));
      k_mmabench<<<1, 128, smem>>>(n, mode, d_out, d_err, 1, 32);
      cudaError_t e = cudaDeviceSynchronize();
      if (e != cudaSuccess) { printf("cuda error %s\n", cudaGetErrorString(e)); return 1; }
      unsigned long long h[8]; uint32_t herr;
      cudaMemcpy(h, d_out, sizeof(h), cudaMemcpyDeviceToHost);
      cudaMemcpy(&herr, d_err, 4, cudaMemcpyDeviceToHost);
      if (r == 1)
        printf("tf32 M128 N32  K8, 1 issuer, %s: %.1f cyc/MMA; err %u\n",
               mode == 2 ? "same tiles every MMA" : "fences + commit every 4 MMAs",
               (double)h[1] / n, herr);
    }
  return 0;
}
