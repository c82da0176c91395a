// Test-infrastructure stub, written for this project (not part of sputnik).
// The reference extension includes sputnik's headers unconditionally but the
// sputnik submodule is not vendored. Only its competitor-baseline entry point
// needs the symbol; the stub makes that entry point report "not supported".
#pragma once
#include <cuda_runtime.h>
namespace sputnik {
inline cudaError_t CudaSpmm(int, int, int, int, const int*, const float*,
                            const int*, const int*, const float*, float*,
                            cudaStream_t) {
  return cudaErrorNotSupported;
}
}  // namespace sputnik
