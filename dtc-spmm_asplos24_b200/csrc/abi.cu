// C-ABI entry points of libdtcspmm.so (declared in include/dtc_spmm.h):
// argument checks, status/error text, per-device state, dispatch.
#include <mutex>
#include <string>
#include <cudaTypedefs.h>
#include "impl.h"

namespace dtc {

namespace {
thread_local std::string g_last_error;
__device__ uint32_t g_device_error;
constexpr int kMaxDev = 64;
std::mutex g_mu;
int g_sms[kMaxDev] = {};
int g_major[kMaxDev] = {};
uint32_t* g_err_ptr[kMaxDev] = {};
uint64_t* g_timer[kMaxDev] = {};
int32_t g_timer_cap[kMaxDev] = {};

int cur_dev() {
  int d = 0;
  cudaGetDevice(&d);
  return d & (kMaxDev - 1);
}

void fill_dev_props(int d) {
  if (g_sms[d]) return;
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
  g_sms[d] = v > 0 ? v : 1;
  cudaDeviceGetAttribute(&v, cudaDevAttrComputeCapabilityMajor, d);
  g_major[d] = v;
}
}  // namespace

void set_error(const std::string& msg) { g_last_error = msg; }

dtc_status cuda_status(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return DTC_ERR_CUDA;
}

int num_sms() {
  int d = cur_dev();
  std::lock_guard<std::mutex> lk(g_mu);
  fill_dev_props(d);
  return g_sms[d];
}

bool is_sm100() {
  int d = cur_dev();
  std::lock_guard<std::mutex> lk(g_mu);
  fill_dev_props(d);
  return g_major[d] == 10;
}

dtc_status encode_c_map(CUtensorMap* map, float* C, int64_t M, int32_t N, int box_rows) {
  static PFN_cuTensorMapEncodeTiled encode = nullptr;
  static std::once_flag once;
  static cudaError_t lookup = cudaSuccess;
  std::call_once(once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    lookup = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (lookup == cudaSuccess && q == cudaDriverEntryPointSuccess)
      encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
  });
  if (!encode) {
    set_error("cuTensorMapEncodeTiled is not available from the driver");
    return DTC_ERR_UNSUPPORTED;
  }
  if (((uintptr_t)C & 15) != 0 || N % 4 != 0 || M < 1 || N < 1) {
    set_error("C must be 16-byte aligned with N % 4 == 0");
    return DTC_ERR_INVALID_ARGUMENT;
  }
  const cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)M};
  const cuuint64_t strides[1] = {(cuuint64_t)N * sizeof(float)};
  const cuuint32_t box[2] = {32u, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1u, 1u};
  CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, C, dims, strides, box, estr,
                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                      CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed for C (code " + std::to_string((int)r) + ")");
    return DTC_ERR_CUDA;
  }
  return DTC_OK;
}

uint64_t* cta_timer_buffer(int32_t* capacity) {
  int d = cur_dev();
  std::lock_guard<std::mutex> lk(g_mu);
  *capacity = g_timer_cap[d];
  return g_timer[d];
}

// The chunk-queue region at byte `offset` of a caller workspace of `bytes`
// bytes, or null when it does not fit (the kernels then run one CTA per chunk).
void* queue_region(void* ws, size_t bytes, size_t offset, int64_t T, int grid) {
  if (!ws) return nullptr;
  const size_t need = spmm_queue_bytes(T, grid);
  char* q = (char*)ws + offset;
  if (((uintptr_t)q & 255) != 0 || offset + need > bytes) return nullptr;
  return q;
}

uint32_t* device_error_word() {
  int d = cur_dev();
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_err_ptr[d]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_device_error) == cudaSuccess) g_err_ptr[d] = (uint32_t*)p;
  }
  return g_err_ptr[d];
}

}  // namespace dtc

using namespace dtc;

extern "C" {

const char* dtc_last_error(void) { return g_last_error.c_str(); }

int dtc_version(void) { return 100; }

/* Reads (and optionally clears) the device-side error word: bit 0 = a
 * bounded wait gave up, bit 1 = an out-of-range index was skipped.
 * Synchronises the device. */
dtc_status dtc_device_status(uint32_t* flags, int clear) {
  DTC_REQUIRE(flags != nullptr, "flags is null");
  uint32_t* p = device_error_word();
  if (!p) { set_error("device error word unavailable"); return DTC_ERR_CUDA; }
  DTC_CUDA(cudaDeviceSynchronize());
  DTC_CUDA(cudaMemcpy(flags, p, 4, cudaMemcpyDeviceToHost));
  if (clear) DTC_CUDA(cudaMemset(p, 0, 4));
  return DTC_OK;
}

dtc_status dtc_set_cta_timer(uint64_t* d_records, int32_t capacity) {
  DTC_REQUIRE(capacity >= 0, "capacity must be >= 0");
  DTC_REQUIRE(capacity == 0 || d_records != nullptr, "null record buffer");
  int d = cur_dev();
  std::lock_guard<std::mutex> lk(g_mu);
  g_timer[d] = capacity > 0 ? d_records : nullptr;
  g_timer_cap[d] = capacity;
  return DTC_OK;
}

dtc_status dtc_rowid_to_window_offset(const int32_t* d_tcblockRowid, int64_t num_blocks,
                                      int32_t num_windows, int32_t* d_rowWindowOffset,
                                      dtc_stream_t stream) {
  DTC_REQUIRE(num_blocks >= 0 && num_windows >= 0, "bad sizes");
  DTC_REQUIRE(d_rowWindowOffset != nullptr, "null rowWindowOffset");
  DTC_REQUIRE(num_blocks == 0 || d_tcblockRowid != nullptr, "null tcblockRowid");
  return rowid_to_rwo(d_tcblockRowid, num_blocks, num_windows, d_rowWindowOffset,
                      (cudaStream_t)stream);
}

dtc_status dtc_spmm(const int32_t* d_rowWindowOffset, const uint8_t* d_tileId,
                    const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                    const float* d_tcValues, int32_t num_nodes, int32_t num_windows,
                    int64_t num_blocks, const float* d_B, int32_t N, float* d_C,
                    dtc_stream_t stream) {
  DTC_REQUIRE(d_rowWindowOffset && d_tcblockOffset && d_B && d_C, "null device pointer");
  DTC_REQUIRE(num_blocks == 0 || (d_tileId && d_sparseAToX), "null device pointer");
  if (N % 4 != 0)
    return spmm_mma_sync_impl(d_rowWindowOffset, d_tileId, d_tcblockOffset, d_sparseAToX,
                              d_tcValues, num_nodes, num_windows, d_B, N, d_C,
                              (cudaStream_t)stream);
  return spmm_tf32_impl(d_rowWindowOffset, d_tileId, d_tcblockOffset, d_sparseAToX, d_tcValues,
                        num_nodes, num_windows, num_blocks, d_B, N, d_C, 0, 0, nullptr,
                        (cudaStream_t)stream);
}

dtc_status dtc_spmm_balance_workspace_bytes(int32_t num_nodes, int64_t num_blocks, int32_t N,
                                            size_t* bytes) {
  DTC_REQUIRE(bytes != nullptr, "bytes is null");
  DTC_REQUIRE(num_nodes >= 0 && num_blocks >= 0 && N >= 1, "bad sizes");
  int32_t nwin = (num_nodes + 15) / 16;
  *bytes = align_up((size_t)(nwin + 1) * 4, 256) + align_up(spmm_partials_bytes(num_blocks, N, 0), 256) +
           spmm_queue_bytes(num_blocks, 0);
  return DTC_OK;
}

dtc_status dtc_spmm_balance(const int32_t* d_tcblockRowid, const uint8_t* d_tileId,
                            const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                            const float* d_tcValues, int32_t num_nodes, int64_t num_blocks,
                            const float* d_B, int32_t N, float* d_C, void* d_workspace,
                            size_t workspace_bytes, dtc_stream_t stream) {
  DTC_REQUIRE(num_nodes >= 0 && num_blocks >= 0 && N >= 1, "bad sizes");
  DTC_REQUIRE(d_tcblockOffset && d_B && d_C, "null device pointer");
  DTC_REQUIRE(num_blocks == 0 || (d_tcblockRowid && d_tileId && d_sparseAToX),
              "null device pointer");
  int32_t nwin = (num_nodes + 15) / 16;
  const size_t rwo_bytes = align_up((size_t)(nwin + 1) * 4, 256);
  const size_t part_bytes = align_up(spmm_partials_bytes(num_blocks, N, 0), 256);
  if (!d_workspace || workspace_bytes < rwo_bytes + part_bytes) {
    set_error("balance workspace too small (dtc_spmm_balance_workspace_bytes)");
    return DTC_ERR_WORKSPACE_TOO_SMALL;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int32_t* rwo = (int32_t*)d_workspace;
  float* part = (float*)((char*)d_workspace + rwo_bytes);
  void* queue = queue_region(d_workspace, workspace_bytes, rwo_bytes + part_bytes, num_blocks, 0);
  dtc_status s = rowid_to_rwo(d_tcblockRowid, num_blocks, nwin, rwo, st);
  if (s != DTC_OK) return s;
  if (N % 4 != 0)
    return spmm_mma_sync_impl(rwo, d_tileId, d_tcblockOffset, d_sparseAToX, d_tcValues,
                              num_nodes, nwin, d_B, N, d_C, st);
  return spmm_tf32_impl(rwo, d_tileId, d_tcblockOffset, d_sparseAToX, d_tcValues, num_nodes,
                        nwin, num_blocks, d_B, N, d_C, 1, 0, part, st, 0, Epilogue{}, 16, queue);
}

dtc_status dtc_spmm_ex_workspace_bytes(int32_t num_nodes, int64_t num_blocks, int32_t N,
                                       int32_t block_h, int mode, int grid, size_t* bytes) {
  DTC_REQUIRE(bytes != nullptr, "bytes is null");
  DTC_REQUIRE(num_nodes >= 0 && num_blocks >= 0 && N >= 1, "bad sizes");
  DTC_REQUIRE(block_h == 16 || block_h == 32, "block_h must be 16 or 32");
  *bytes = ((mode == 1) ? align_up(spmm_partials_bytes(num_blocks, N, grid, block_h), 256) : 0) +
           spmm_queue_bytes(num_blocks, grid);
  return DTC_OK;
}

}  // extern "C"

namespace {

dtc_status spmm_ex_impl(const int32_t* rwo, const uint8_t* tile, const int32_t* toff,
                        const int32_t* s2x, const float* vals, int32_t M, int32_t nwin, int64_t T,
                        int32_t H, int32_t W, int bformat, const void* p0, const void* p1, int32_t N,
                        int precision, float* C, int mode, int grid, int ntile, Epilogue epi,
                        void* ws, size_t wsb, cudaStream_t st) {
  DTC_REQUIRE(mode == 0 || mode == 1, "mode must be 0 (window) or 1 (balance)");
  DTC_REQUIRE(grid >= 0, "grid must be >= 0");
  DTC_REQUIRE(ntile == 0 || ntile == 1 || ntile == 2 || ntile == 4, "ntile must be 0, 1, 2 or 4");
  DTC_REQUIRE(rwo && toff && p0 && C, "null device pointer");
  DTC_REQUIRE(M >= 0 && T >= 0 && N >= 1, "bad sizes");
  DTC_REQUIRE(H == 16 || H == 32, "block_h must be 16 or 32");
  // required: the partial tiles of balance mode; optional after them: the
  // chunk queue (persistent CTAs)
  const size_t part_bytes = (mode == 1) ? align_up(spmm_partials_bytes(T, N, grid, H), 256) : 0;
  if (part_bytes > 0 && (!ws || wsb < part_bytes)) {
    set_error("spmm workspace too small (dtc_spmm_ex_workspace_bytes)");
    return DTC_ERR_WORKSPACE_TOO_SMALL;
  }
  void* queue = queue_region(ws, wsb, part_bytes, T, grid);
  if (bformat == DTC_B_F32 && precision == DTC_PREC_TF32)
    return spmm_tf32_impl(rwo, tile, toff, s2x, vals, M, nwin, T, (const float*)p0, N, C, mode,
                          grid, (float*)ws, st, ntile, epi, H, queue, W);
  return spmm_split_impl(rwo, tile, toff, s2x, vals, M, nwin, T, bformat, p0, p1, N, precision,
                         C, mode, grid, (float*)ws, st, ntile, epi, H, queue, W);
}

}  // namespace

extern "C" {

dtc_status dtc_spmm_ex(const int32_t* d_rowWindowOffset, const uint8_t* d_tileId,
                       const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                       const float* d_tcValues, int32_t num_nodes, int32_t num_windows,
                       int64_t num_blocks, int32_t block_h, int32_t block_w, int bformat,
                       const void* d_Bplane0, const void* d_Bplane1, int32_t N, int precision,
                       float* d_C, int mode, int grid, int ntile, void* d_workspace,
                       size_t workspace_bytes, dtc_stream_t stream) {
  return spmm_ex_impl(d_rowWindowOffset, d_tileId, d_tcblockOffset, d_sparseAToX, d_tcValues,
                      num_nodes, num_windows, num_blocks, block_h, block_w, bformat, d_Bplane0,
                      d_Bplane1, N,
                      precision, d_C, mode, grid, ntile, Epilogue{}, d_workspace,
                      workspace_bytes, (cudaStream_t)stream);
}

dtc_status dtc_spmm_fused(const int32_t* d_rowWindowOffset, const uint8_t* d_tileId,
                          const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                          const float* d_tcValues, int32_t num_nodes, int32_t num_windows,
                          int64_t num_blocks, int32_t block_h, int32_t block_w, int bformat,
                          const void* d_Bplane0, const void* d_Bplane1, int32_t N,
                          int precision, const float* d_bias,
                          int relu, float* d_C, int mode, int grid, int ntile, void* d_workspace,
                          size_t workspace_bytes, dtc_stream_t stream) {
  Epilogue e;
  e.bias = d_bias;
  e.relu = relu != 0;
  return spmm_ex_impl(d_rowWindowOffset, d_tileId, d_tcblockOffset, d_sparseAToX, d_tcValues,
                      num_nodes, num_windows, num_blocks, block_h, block_w, bformat, d_Bplane0,
                      d_Bplane1, N, precision, d_C, mode, grid, ntile, e, d_workspace,
                      workspace_bytes,
                      (cudaStream_t)stream);
}

dtc_status dtc_spmm_mma_sync(const int32_t* d_rowWindowOffset, const uint8_t* d_tileId,
                             const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                             const float* d_tcValues, int32_t num_nodes, int32_t num_windows,
                             const float* d_B, int32_t N, float* d_C, dtc_stream_t stream) {
  DTC_REQUIRE(d_rowWindowOffset && d_tcblockOffset && d_B && d_C, "null device pointer");
  return spmm_mma_sync_impl(d_rowWindowOffset, d_tileId, d_tcblockOffset, d_sparseAToX,
                            d_tcValues, num_nodes, num_windows, d_B, N, d_C,
                            (cudaStream_t)stream);
}

dtc_status dtc_bformat_bytes(int fmt, int64_t rows, int32_t N, size_t* plane0, size_t* plane1) {
  return bformat_bytes_impl(fmt, rows, N, plane0, plane1);
}

dtc_status dtc_pack_b(int fmt, const float* d_B, int64_t rows, int32_t N, void* d_plane0,
                      void* d_plane1, dtc_stream_t stream) {
  return pack_b_impl(fmt, d_B, rows, N, d_plane0, d_plane1, (cudaStream_t)stream);
}

}  // extern "C"
