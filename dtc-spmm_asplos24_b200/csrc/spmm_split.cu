// Split-precision TC-block SpMM (bf16 hi/lo products on tcgen05 kind::f16).
#include "common.cuh"

namespace dtc {

dtc_status spmm_split_impl(const int32_t*, const uint8_t*, const int32_t*, const int32_t*,
                           const float*, int32_t, int32_t, int64_t, int, const void*, const void*,
                           int32_t, int, float*, int, int, float*, cudaStream_t) {
  set_error("split-precision forms are not built yet");
  return DTC_ERR_UNSUPPORTED;
}

}  // namespace dtc
