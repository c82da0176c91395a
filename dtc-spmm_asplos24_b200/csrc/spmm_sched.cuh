// Scheduling pieces shared by the TC-block SpMM kernels (tf32 and split
// precision): kernel parameters, CTA block ranges, the window walk, the
// A-tile layout, cp.async helpers and the deterministic partial reduction.
#pragma once
#include "common.cuh"

namespace dtc {
namespace {

// Default CTA count: the kernels hold one CTA per SM (shared memory), so 16
// CTAs per SM run as 16 waves; a CTA that finishes early picks up the next
// range, which evens out the per-range cost differences of skewed matrices.
constexpr int kWavesPerSm = 16;
inline int default_grid() { return kWavesPerSm * num_sms(); }
constexpr int kBlkW = 8;        // TC-block width (BLK_W)

struct Params {
  CUtensorMap cmap;          // C [M x N] fp32, box 32 columns x window height (TMA stores)
  const int32_t* rwo;        // RowWindowOffset [nwin+1]
  const uint8_t* tile;       // TCblocktileId [nnz]
  const int32_t* toff;       // TCblockoffset [T+1]
  const int32_t* s2x;        // SparseAToX [T*8]
  const float* vals;         // tile-order values or null (A = 1)
  const float* B;            // [M x N] fp32 (tf32 form) / hi or q plane (split forms)
  const void* B1;            // second plane (split forms): ext bytes or fp8 row scales
  int32_t bformat;
  float* C;                  // [M x N]
  float* part;               // partial tiles [2*G x 16 x N] (balance mode)
  uint32_t* err;
  const float* bias;         // epilogue bias [N] or null
  int32_t relu;              // epilogue ReLU
  int32_t M, nwin, N, G, mode;
  int32_t H;                 // row-window height (16 or 32)
  int64_t T;
};

// The epilogue applied to a finished C element of column f.
__device__ __forceinline__ float epilogue(const Params& p, float x, int f) {
  if (p.bias) x += __ldg(p.bias + f);
  return p.relu ? fmaxf(x, 0.0f) : x;
}

__device__ __forceinline__ int32_t lower_bound_i32(const int32_t* a, int32_t n, int64_t x) {
  int32_t lo = 0, hi = n;
  while (lo < hi) {
    int32_t mid = (lo + hi) >> 1;
    if ((int64_t)__ldg(a + mid) < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// CTA block range (see header comment).
__device__ __forceinline__ void cta_range(const Params& p, int c, int64_t& b0, int64_t& b1) {
  b0 = (int64_t)c * p.T / p.G;
  b1 = (int64_t)(c + 1) * p.T / p.G;
  if (p.mode == 0) {  // snap to window starts: windows never split
    int32_t w0 = lower_bound_i32(p.rwo, p.nwin, b0);
    b0 = (w0 < p.nwin) ? __ldg(p.rwo + w0) : p.T;
    if (c + 1 < p.G) {
      int32_t w1 = lower_bound_i32(p.rwo, p.nwin, b1);
      b1 = (w1 < p.nwin) ? __ldg(p.rwo + w1) : p.T;
    } else {
      b1 = p.T;
    }
  }
}

// Windows walked by a CTA: [w_start, w_end). Empty windows in the range are
// owned by this CTA (their C rows are zeroed here); nonempty windows whose
// intersection with [b0, b1) is empty are skipped.
__device__ __forceinline__ void cta_windows(const Params& p, int c, int64_t b0, int64_t b1,
                                            int32_t& w_start, int32_t& w_end) {
  int32_t wl = lower_bound_i32(p.rwo, p.nwin, b0);
  if (wl > 0 && (wl == p.nwin || (int64_t)__ldg(p.rwo + wl) > b0)) wl -= 1;
  w_start = wl;
  w_end = (c + 1 == p.G) ? p.nwin : lower_bound_i32(p.rwo, p.nwin, b1);
}

// Byte offset of A_b^T element (window row r, slot s) in the K-major,
// no-swizzle core-matrix layout (8 rows x 16 B core matrices; LBO = 128 B
// between the two K halves, SBO = 256 B between the two 8-row groups).
__device__ __forceinline__ uint32_t y_offset(uint32_t pos) {
  uint32_t r = pos >> 3, s = pos & 7;
  return (r & 7) * 16 + (r >> 3) * 256 + (s >> 2) * 128 + (s & 3) * 4;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Sums the partial tiles of every window cut by CTA boundaries, in CTA order
// (bitwise reproducible), and writes its C rows. One CTA per boundary.
__global__ void k_reduce_partials(const Params p) {
  const int c = blockIdx.x + 1;  // boundary between CTA c-1 and c
  const int64_t bc = (int64_t)c * p.T / p.G;
  const int64_t bprev = (int64_t)(c - 1) * p.T / p.G;
  // window containing block bc: largest w with rwo[w] <= bc
  int32_t lo = 0, hi = p.nwin;
  while (lo < hi) {
    int32_t mid = (lo + hi + 1) >> 1;
    if (__ldg(p.rwo + mid) <= bc) lo = mid; else hi = mid - 1;
  }
  const int32_t w = lo;
  if (w >= p.nwin) return;
  const int64_t r0 = __ldg(p.rwo + w), r1 = __ldg(p.rwo + w + 1);
  if (!(r0 < bc && bc < r1)) return;           // boundary not inside window w
  if (c - 1 >= 1 && bprev > r0) return;        // an earlier boundary owns it
  // contributors: CTA c-1 (tail slot), CTAs c..c_last (head slots)
  int c_last = c;
  while (c_last + 1 < p.G && (int64_t)(c_last + 1) * p.T / p.G < r1) ++c_last;
  const int64_t row0 = (int64_t)w * p.H;
  const int64_t elems = (int64_t)p.H * p.N;
  for (int64_t x = threadIdx.x; x < elems; x += blockDim.x) {
    const int r = (int)(x / p.N);
    if (row0 + r >= p.M) continue;
    float acc = p.part[(size_t)(2 * (c - 1) + 1) * elems + x];
    for (int k = c; k <= c_last; ++k) acc += p.part[(size_t)(2 * k) * elems + x];
    p.C[row0 * p.N + x] = epilogue(p, acc, (int)(x - (int64_t)r * p.N));
  }
}

}  // namespace
}  // namespace dtc
