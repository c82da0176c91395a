// TC-block SpMM on sm_100a: TMA tile::gather4 of dense rows into 128-byte
// swizzled shared memory, tcgen05.mma into TMEM, warp-specialised persistent
// CTAs, deterministic strict balance.
//
// Product mapping. The reference multiplies each 16x8 TC block A_b (rows of a
// row window x compacted column slots) by the 8 gathered rows of B with
// mma.sync m16n8k8 (DTC-SpMM/DTCSpMM_kernel.cu:2776-2794). tcgen05 needs
// M in {64,128}, so the product is transposed:
//     C_w^T [features x 16] += B_b^T [features x 8] * A_b^T [8 x 16]
// UMMA M = 128 features (one N-tile), N = 16 window rows, K = 8 slots (tf32)
// or 16 (bf16: hi rows + lo rows). Operand "A" of the UMMA is the gathered
// B rows, which land MN-major (features contiguous) straight from the TMA
// gather; operand "B" is the densified TC block, K-major, built by warps.
// kind::tf32 reads an MN-major operand only in the 128-byte swizzle with
// 32-byte granules (layout type 1; 16-byte granules read as zeros), which
// the TMA produces with CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B.
//
// Work split. CTA c owns TC blocks [c*T/G, (c+1)*T/G) (strict balance) or
// that range snapped to row-window starts (window mode). Windows cut by a
// CTA boundary write fp32 partial tiles to a workspace; k_reduce_partials
// sums them in CTA order, so results do not depend on timing.
//
// Warp roles (320 threads):
//   warps 0-3  epilogue: tcgen05.ld 32x32b, coalesced stores of C rows
//   warp  4    producer: SparseAToX prefetch, TMA gather4 issue
//   warp  5    TMEM allocator + single-thread UMMA issuer
//   warps 6-9  tile builders: zero + scatter TC-block values into A_b^T
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include "common.cuh"

namespace dtc {
namespace {

constexpr int kEpiWarps = 4;
constexpr int kProdWarp = 4;
constexpr int kMmaWarp = 5;
constexpr int kTileWarp0 = 6;
constexpr int kTileWarps = 4;
constexpr int kThreads = 32 * (kTileWarp0 + kTileWarps);  // 320
constexpr int kNacc = 4;        // TMEM accumulator buffers in flight
constexpr int kWinH = 16;       // row-window height (BLK_H)
constexpr int kBlkW = 8;        // TC-block width (BLK_W)
constexpr int kXTileBytes = 4096;   // 8 rows x 128 fp32 features
constexpr int kYBytes = 512;        // 16 x 8 fp32, K-major core matrices

struct Params {
  const int32_t* rwo;        // RowWindowOffset [nwin+1]
  const uint8_t* tile;       // TCblocktileId [nnz]
  const int32_t* toff;       // TCblockoffset [T+1]
  const int32_t* s2x;        // SparseAToX [T*8]
  const float* vals;         // tile-order values or null (A = 1)
  float* C;                  // [M x N]
  float* part;               // partial tiles [2*G x 16 x N] (balance mode)
  uint32_t* err;
  int32_t M, nwin, N, G, mode, nchunks;  // nchunks: 32-feature chunks per CTA slice
  int64_t T;
};

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
// owned by this CTA (their C rows are zeroed here).
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

template <int NT, int S>
struct Smem {
  static constexpr int kX = S * NT * kXTileBytes;
  static constexpr int kY = S * kYBytes;
  static constexpr int kBars = (4 * S + 2 * kNacc) * 8;
  static constexpr int kTotal = kX + kY + kBars + 16 + 1024;  // + alignment slack
};

template <int NT, int S>
__global__ void __launch_bounds__(kThreads, 1)
    k_spmm_tf32(const __grid_constant__ CUtensorMap tmapB, const Params p) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* xring = smem;
  uint8_t* yring = smem + Smem<NT, S>::kX;
  uint64_t* bars = (uint64_t*)(yring + Smem<NT, S>::kY);
  uint64_t* tma_full = bars;            // [S] producer expect_tx + TMA bytes
  uint64_t* tile_full = bars + S;       // [S] one tile-builder arrive
  uint64_t* empty = bars + 2 * S;       // [S] UMMA commit
  uint64_t* acc_full = bars + 4 * S;    // [kNacc] UMMA commit
  uint64_t* acc_empty = acc_full + kNacc;  // [kNacc] 4 epilogue warps
  uint32_t* tmem_slot = (uint32_t*)(acc_empty + kNacc);
  volatile uint32_t* abort_flag = tmem_slot + 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x;
  const int slice = blockIdx.y;               // 128*NT-feature column slice
  const int col0 = slice * NT * 128;
  int nch = p.nchunks - slice * NT * 4;       // chunks in this slice
  if (nch > NT * 4) nch = NT * 4;
  constexpr uint32_t kTmemCols = (kNacc * NT * 16 <= 32) ? 32 : (kNacc * NT * 16 <= 64) ? 64
                                 : (kNacc * NT * 16 <= 128) ? 128 : 256;

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&tma_full[i], 1);
      mbar_init(&tile_full[i], 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < kNacc; ++i) {
      mbar_init(&acc_full[i], 1);
      mbar_init(&acc_empty[i], kEpiWarps);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == kMmaWarp) {
    tmem_alloc(tmem_slot, kTmemCols);
    tmem_relinquish();
  }
  if (warp == kProdWarp && lane == 0) prefetch_tensormap(&tmapB);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  int64_t b0, b1;
  cta_range(p, c, b0, b1);
  const int64_t nblk = b1 - b0;

  if (warp == kProdWarp) {
    // ---------------------------------------------------------------- TMA
    const uint32_t bytes = (uint32_t)nch * 2u * 512u;
    int4 rows_lo = make_int4(0, 0, 0, 0), rows_hi = rows_lo;  // block b0+32g+lane
    int4 nxt_lo = rows_lo, nxt_hi = rows_lo;
    auto load_group = [&](int64_t g, int4& lo, int4& hi) {
      int64_t b = b0 + g * 32 + lane;
      if (b < b1) {
        const int4* q = reinterpret_cast<const int4*>(p.s2x + b * kBlkW);
        lo = __ldg(q);
        hi = __ldg(q + 1);
      }
    };
    if (nblk > 0) load_group(0, nxt_lo, nxt_hi);
    for (int64_t i = 0; i < nblk; ++i) {
      const int j = (int)(i & 31);
      if (j == 0) {
        rows_lo = nxt_lo;
        rows_hi = nxt_hi;
        if (i + 32 < nblk) load_group((i >> 5) + 1, nxt_lo, nxt_hi);
      }
      const int s = (int)(i % S);
      const uint32_t n = (uint32_t)(i / S);
      const bool got = mbar_wait(&empty[s], (n & 1) ^ 1, p.err);
      if (!__all_sync(0xffffffffu, got) || *abort_flag) { *abort_flag = 1; break; }
      int32_t r[8];
      r[0] = __shfl_sync(0xffffffffu, rows_lo.x, j);
      r[1] = __shfl_sync(0xffffffffu, rows_lo.y, j);
      r[2] = __shfl_sync(0xffffffffu, rows_lo.z, j);
      r[3] = __shfl_sync(0xffffffffu, rows_lo.w, j);
      r[4] = __shfl_sync(0xffffffffu, rows_hi.x, j);
      r[5] = __shfl_sync(0xffffffffu, rows_hi.y, j);
      r[6] = __shfl_sync(0xffffffffu, rows_hi.z, j);
      r[7] = __shfl_sync(0xffffffffu, rows_hi.w, j);
      // padded slots (always after slot 0, column id 0) -> out-of-range row: zero fill
#pragma unroll
      for (int k = 1; k < 8; ++k)
        if (r[k] == 0) r[k] = p.M;
      if (lane == 0) mbar_arrive_expect_tx(&tma_full[s], bytes);
      __syncwarp();
      uint8_t* xs = xring + (size_t)s * NT * kXTileBytes;
      for (int o = lane; o < 2 * nch; o += 32) {
        const int h = o & 1, ch = o >> 1;
        uint8_t* dst = xs + ch * 1024 + h * 512;
        tma_gather4(dst, &tmapB, &tma_full[s], col0 + ch * 32, r[4 * h + 0], r[4 * h + 1],
                    r[4 * h + 2], r[4 * h + 3]);
      }
    }
  } else if (warp >= kTileWarp0) {
    // ------------------------------------------------------ tile builders
    // Warp tw owns ring stages [tw*kBatch, (tw+1)*kBatch) in every round, so
    // each warp waits on its stages' `empty` phases strictly in order (a
    // parity wait more than one phase ahead would pass spuriously).
    constexpr int kBatch = S / kTileWarps;
    static_assert(S % kTileWarps == 0 && kBatch >= 1 && kBatch <= 31, "ring split");
    const int tw = warp - kTileWarp0;
    for (int64_t bb = b0 + (int64_t)tw * kBatch; bb < b1; bb += (int64_t)S) {
      const int nb = (int)((b1 - bb) < kBatch ? (b1 - bb) : kBatch);
      int32_t offv = (lane <= nb) ? __ldg(p.toff + bb + lane) : 0;
      int32_t off[kBatch + 1];
#pragma unroll
      for (int k = 0; k <= kBatch; ++k) off[k] = __shfl_sync(0xffffffffu, offv, k);
      // wait for the batch's stages, zero their A tiles
      bool ok = true;
      for (int k = 0; k < nb; ++k) {
        const int64_t i = bb + k - b0;
        const int s = (int)(i % S);
        const uint32_t n = (uint32_t)(i / S);
        const bool got = mbar_wait(&empty[s], (n & 1) ^ 1, p.err);
        if (!__all_sync(0xffffffffu, got)) { ok = false; break; }
        float4* y = reinterpret_cast<float4*>(yring + (size_t)s * kYBytes);
        y[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      if (!__all_sync(0xffffffffu, ok && !*abort_flag)) { *abort_flag = 1; break; }
      const int32_t e0 = off[0], e1 = off[nb];
      for (int32_t e = e0 + lane; e < e1; e += 32) {
        int k = 0;
#pragma unroll
        for (int q = 1; q < kBatch; ++q) k += (q < nb && e >= off[q]) ? 1 : 0;
        const uint32_t pos = __ldg(p.tile + e);
        float v = p.vals ? __ldg(p.vals + e) : 1.0f;
        if (pos < kWinH * kBlkW && v != 0.0f) {
          uint32_t t32;
          asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t32) : "f"(v));
          const int s = (int)((bb + k - b0) % S);
          *reinterpret_cast<uint32_t*>(yring + (size_t)s * kYBytes + y_offset(pos)) = t32;
        } else if (pos >= kWinH * kBlkW) {
          atomicOr(p.err, kErrBadIndex);
        }
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0)
        for (int k = 0; k < nb; ++k) mbar_arrive(&tile_full[(int)((bb + k - b0) % S)]);
    }
  } else if (warp == kMmaWarp) {
    // ------------------------------------------------------------- UMMA
    if (lane == 0) {
      int32_t ws, we;
      cta_windows(p, c, b0, b1, ws, we);
      constexpr uint32_t idesc = umma_idesc(2, 128, 16, 1, 0);
      const uint32_t xbase = smem_u32(xring), ybase = smem_u32(yring);
      int64_t i = 0;  // block counter within the CTA range
      uint32_t q = 0;  // segment counter
      bool ok = true;
      for (int32_t w = ws; w < we && ok; ++w) {
        const int64_t r0 = __ldg(p.rwo + w), r1 = __ldg(p.rwo + w + 1);
        if (r0 == r1) continue;
        const int64_t s0 = r0 > b0 ? r0 : b0, s1 = r1 < b1 ? r1 : b1;
        const int a = (int)(q % kNacc);
        if (!mbar_wait(&acc_empty[a], ((q / kNacc) & 1) ^ 1, p.err)) { ok = false; break; }
        tc_fence_after();
        for (int64_t b = s0; b < s1; ++b, ++i) {
          const int s = (int)(i % S);
          const uint32_t n = (uint32_t)(i / S);
          if (!mbar_wait(&tma_full[s], n & 1, p.err) || !mbar_wait(&tile_full[s], n & 1, p.err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint64_t bdesc = umma_desc(ybase + s * kYBytes, 128, 256, 0);
#pragma unroll
          for (int t = 0; t < NT; ++t) {
            // MN-major tf32 operands use the 128-byte swizzle with 32-byte
            // granules (UMMA layout type 1): atoms of 32 features x 4 rows;
            // LBO = 1024 B between 32-feature atoms, SBO = 512 B between the
            // two 4-row halves -- exactly where the two gather4 ops land.
            const uint64_t adesc = umma_desc(xbase + (s * NT + t) * kXTileBytes, 1024, 512, 1);
            mma_tf32(tmem_base + (uint32_t)((a * NT + t) * 16), adesc, bdesc, idesc,
                     b == s0 ? 0u : 1u);
          }
          tc_commit(&empty[s]);
        }
        if (!ok) break;
        tc_commit(&acc_full[a]);
        ++q;
      }
      if (!ok) *abort_flag = 1;
    }
    __syncwarp();
  } else {
    // --------------------------------------------------------- epilogue
    int32_t ws, we;
    cta_windows(p, c, b0, b1, ws, we);
    const int ew = warp;  // TMEM lanes 32*ew .. 32*ew+31
    uint32_t q = 0;
    for (int32_t w = ws; w < we; ++w) {
      const int64_t r0 = __ldg(p.rwo + w), r1 = __ldg(p.rwo + w + 1);
      const int64_t row0 = (int64_t)w * kWinH;
      if (r0 == r1) {  // empty window: C rows are zero
        for (int f = col0 + ew * 32 + lane; f < p.N && f < col0 + NT * 128; f += 128)
          for (int r = 0; r < kWinH && row0 + r < p.M; ++r) p.C[(row0 + r) * p.N + f] = 0.0f;
        continue;
      }
      const int a = (int)(q % kNacc);
      const bool got = mbar_wait(&acc_full[a], (q / kNacc) & 1, p.err);
      if (!__all_sync(0xffffffffu, got)) { *abort_flag = 1; break; }
      tc_fence_after();
      float* out;
      int64_t ld;
      bool guard_rows = true;
      if (p.mode == 1 && (r0 < b0 || r1 > b1)) {  // window cut by a CTA boundary
        const int slot = (r0 < b0) ? 2 * c : 2 * c + 1;
        out = p.part + (size_t)slot * kWinH * p.N;
        guard_rows = false;
      } else {
        out = p.C + row0 * p.N;
      }
      ld = p.N;
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        uint32_t v[16];
        tmem_ld16(tmem_base + ((uint32_t)(ew * 32) << 16) + (uint32_t)((a * NT + t) * 16), v);
        tmem_ld_wait();
        const int f = col0 + t * 128 + ew * 32 + lane;
        if (t == NT - 1) {
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[a]);
        }
        if (f < p.N) {
#pragma unroll
          for (int r = 0; r < kWinH; ++r)
            if (!guard_rows || row0 + r < p.M) out[r * ld + f] = __uint_as_float(v[r]);
        }
      }
      ++q;
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    tmem_dealloc(tmem_base, kTmemCols);
  }
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
  const int64_t row0 = (int64_t)w * kWinH;
  const int64_t elems = (int64_t)kWinH * p.N;
  for (int64_t x = threadIdx.x; x < elems; x += blockDim.x) {
    const int r = (int)(x / p.N);
    if (row0 + r >= p.M) continue;
    float acc = p.part[(size_t)(2 * (c - 1) + 1) * elems + x];
    for (int k = c; k <= c_last; ++k) acc += p.part[(size_t)(2 * k) * elems + x];
    p.C[row0 * p.N + x] = acc;
  }
}

__global__ void k_rowid_to_rwo(const int32_t* __restrict__ rowid, int64_t T, int32_t nwin,
                               int32_t* __restrict__ rwo) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b <= T; b += stride) {
    const int32_t prev = (b == 0) ? -1 : __ldg(rowid + b - 1);
    const int32_t cur = (b == T) ? nwin : __ldg(rowid + b);
    for (int32_t w = prev + 1; w <= cur; ++w) rwo[w] = (int32_t)b;
  }
}

PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* ptr = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)ptr;
  }
  return fn;
}

// 2-D map over a row-major [rows x N] matrix of `esize`-byte elements, box =
// 128 bytes x 1 row, 128-byte swizzle. 4-byte elements use 32-byte swizzle
// granules (the layout UMMA kind::tf32 reads MN-major), 2-byte elements the
// 16-byte granules of the standard 128-byte swizzle.
dtc_status make_row_map(CUtensorMap* map, const void* base, CUtensorMapDataType dt, int esize,
                        int64_t rows, int32_t N) {
  auto enc = get_encode();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return DTC_ERR_UNSUPPORTED;
  }
  cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)N * esize};
  cuuint32_t box[2] = {(cuuint32_t)(128 / esize), 1};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, dt, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE,
                   esize == 4 ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B : CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return DTC_ERR_CUDA;
  }
  return DTC_OK;
}

template <int NT, int S>
dtc_status launch_tf32(const CUtensorMap& map, const Params& p, int slices, cudaStream_t st) {
  constexpr int smem = Smem<NT, S>::kTotal;
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    DTC_CUDA(cudaFuncSetAttribute(k_spmm_tf32<NT, S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  smem));
    attr_set[dev & 63] = true;
  }
  dim3 grid((unsigned)p.G, (unsigned)slices);
  k_spmm_tf32<NT, S><<<grid, kThreads, smem, st>>>(map, p);
  DTC_CUDA(cudaGetLastError());
  if (p.mode == 1 && p.G > 1) {
    k_reduce_partials<<<p.G - 1, 256, 0, st>>>(p);
    DTC_CUDA(cudaGetLastError());
  }
  return DTC_OK;
}

}  // namespace

// Shared implementation behind dtc_spmm / dtc_spmm_balance / dtc_spmm_ex (fp32 B).
dtc_status spmm_tf32_impl(const int32_t* rwo, const uint8_t* tile, const int32_t* toff,
                          const int32_t* s2x, const float* vals, int32_t M, int32_t nwin,
                          int64_t T, const float* B, int32_t N, float* C, int mode, int grid,
                          float* part, cudaStream_t st) {
  DTC_REQUIRE(M >= 0 && N >= 1 && T >= 0, "bad sizes");
  DTC_REQUIRE(N % 4 == 0, "tcgen05 path needs N % 4 == 0 (16-byte TMA row stride)");
  DTC_REQUIRE(((uintptr_t)B & 15) == 0, "B must be 16-byte aligned");
  DTC_REQUIRE(nwin == (M + kWinH - 1) / kWinH, "num_windows must be ceil(num_nodes/16)");
  if (!is_sm100()) {
    set_error("tcgen05 kernels need an sm_100 device");
    return DTC_ERR_UNSUPPORTED;
  }
  if (M == 0) return DTC_OK;
  if (T == 0) {
    DTC_CUDA(cudaMemsetAsync(C, 0, (size_t)M * N * sizeof(float), st));
    return DTC_OK;
  }
  Params p{};
  p.rwo = rwo; p.tile = tile; p.toff = toff; p.s2x = s2x; p.vals = vals;
  p.C = C; p.part = part; p.err = device_error_word();
  p.M = M; p.nwin = nwin; p.N = N; p.T = T; p.mode = mode;
  int G = grid > 0 ? grid : num_sms();
  if ((int64_t)G > T) G = (int)T;
  p.G = G;
  p.nchunks = (N + 31) / 32;
  CUtensorMap map;
  dtc_status s = make_row_map(&map, B, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, M, N);
  if (s != DTC_OK) return s;
  if (N <= 128) return launch_tf32<1, 32>(map, p, 1, st);
  if (N <= 256) return launch_tf32<2, 24>(map, p, 1, st);
  return launch_tf32<4, 12>(map, p, (N + 511) / 512, st);
}

size_t spmm_partials_bytes(int64_t T, int32_t N, int grid) {
  int G = grid > 0 ? grid : num_sms();
  if ((int64_t)G > T) G = (int)(T > 0 ? T : 1);
  return (size_t)2 * G * kWinH * (size_t)N * sizeof(float);
}

dtc_status rowid_to_rwo(const int32_t* rowid, int64_t T, int32_t nwin, int32_t* rwo,
                        cudaStream_t st) {
  int64_t n = T + 1;
  unsigned g = (unsigned)((n + 255) / 256);
  if (g > 65535u * 16) g = 65535u * 16;
  k_rowid_to_rwo<<<g, 256, 0, st>>>(rowid, T, nwin, rwo);
  DTC_CUDA(cudaGetLastError());
  return DTC_OK;
}

}  // namespace dtc
