// Strict-balance SpMM for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a serving process that has handed all
// device memory to its own budgeted pool, plugins whose host forbids
// allocations on the hot path, and plain-C users without an allocator. The
// regular strict-balance entry point (dtc_spmm_balance) needs a caller-sized
// workspace for its window-offset table and per-CTA partial tiles; this
// variant keeps that scratch in a fixed array inside the library instead.
//
// The array lives in device memory of every GPU that loads the library and
// stays allocated until the process exits. Its first use on a device looks up
// the array's device address (cudaGetSymbolAddress) with that device current;
// make that first call before any stream capture. All calls share the array,
// so two calls that overlap on the GPU (different streams, or different host
// threads on the same device) race on it and must be serialised by the
// caller. Nothing in the array needs to start at zero: every byte a call reads
// was written earlier in the same call.
#include <mutex>
#include "impl.h"


namespace {

constexpr size_t kScratchBytes = 16u << 20;  // 16 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_ptr[64] = {};

// Device address of the scratch array on the current device (looked up once
// per device, with that device current).
dtc_status scratch_address(void** out) {
  int dev = 0;
  DTC_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    dtc::set_error("device ordinal out of range for the no-alloc scratch table");
    return DTC_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return dtc::cuda_status(e != cudaSuccess ? e : cudaErrorInvalidSymbol,
                              "cudaGetSymbolAddress(no-alloc scratch)");
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return DTC_OK;
}

}  // namespace

extern "C" size_t dtc_noalloc_scratch_capacity(void) { return kScratchBytes; }

extern "C" dtc_status dtc_spmm_balance_noalloc(const int32_t* d_tcblockRowid,
                                               const uint8_t* d_tileId,
                                               const int32_t* d_tcblockOffset,
                                               const int32_t* d_sparseAToX,
                                               const float* d_tcValues, int32_t num_nodes,
                                               int64_t num_blocks, const float* d_B, int32_t N,
                                               float* d_C, dtc_stream_t stream) {
  using namespace dtc;
  DTC_REQUIRE(num_nodes >= 0 && num_blocks >= 0 && N >= 1, "bad sizes");
  DTC_REQUIRE(d_tcblockOffset && d_B && d_C, "null device pointer");
  DTC_REQUIRE(num_blocks == 0 || (d_tcblockRowid && d_tileId && d_sparseAToX),
              "null device pointer");
  const int32_t nwin = (num_nodes + 15) / 16;
  // one CTA per SM keeps the partial tiles small: 2 slots x 16 rows x N per CTA
  int grid = num_sms();
  if ((int64_t)grid > num_blocks) grid = (int)(num_blocks > 0 ? num_blocks : 1);
  const size_t rwo_bytes = align_up((size_t)(nwin + 1) * 4, 256);
  const size_t part_bytes = (N % 4 == 0) ? (size_t)2 * grid * 16 * (size_t)N * 4 : 0;
  if (rwo_bytes + part_bytes > kScratchBytes) {
    set_error("dtc_spmm_balance_noalloc: needs " + std::to_string(rwo_bytes + part_bytes) +
              " bytes of scratch (4*(ceil(num_nodes/16)+1) rounded to 256, plus 128*N per SM) "
              "but the built-in array holds " + std::to_string(kScratchBytes) +
              "; use dtc_spmm_balance with a caller workspace");
    return DTC_ERR_WORKSPACE_TOO_SMALL;
  }
  void* base = nullptr;
  dtc_status s = scratch_address(&base);
  if (s != DTC_OK) return s;
  cudaStream_t st = (cudaStream_t)stream;
  int32_t* rwo = (int32_t*)base;
  float* part = (float*)((char*)base + rwo_bytes);
  s = rowid_to_rwo(d_tcblockRowid, num_blocks, nwin, rwo, st);
  if (s != DTC_OK) return s;
  if (N % 4 != 0)
    return spmm_mma_sync_impl(rwo, d_tileId, d_tcblockOffset, d_sparseAToX, d_tcValues,
                              num_nodes, nwin, d_B, N, d_C, st);
  return spmm_tf32_impl(rwo, d_tileId, d_tcblockOffset, d_sparseAToX, d_tcValues, num_nodes,
                        nwin, num_blocks, d_B, N, d_C, 1, grid, part, st);
}
