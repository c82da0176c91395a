// TC-block SpMM on sm_100a: cp.async gathers of dense rows into swizzled
// shared memory, tcgen05.mma into TMEM, warp-specialised persistent CTAs,
// deterministic strict balance.
//
// Product mapping. The reference multiplies each 16x8 TC block A_b (rows of a
// row window x compacted column slots) by the 8 gathered rows of B with
// mma.sync m16n8k8 (DTC-SpMM/DTCSpMM_kernel.cu:2776-2794). tcgen05 needs
// M in {64,128}, so the product is transposed:
//     C_w^T [features x 16] += B_b^T [features x 8] * A_b^T [8 x 16]
// UMMA M = 128 features (one N-tile), N = 16 window rows, K = 8 slots. The
// UMMA "A" operand is the gathered B rows, stored MN-major (features
// contiguous); the UMMA "B" operand is the densified TC block, K-major.
// kind::tf32 reads an MN-major operand only in the 128-byte swizzle with
// 32-byte granules (UMMA layout type 1: atoms of 32 features x 4 rows; with
// 16-byte granules it reads zeros); the loaders write that layout directly.
//
// Work split. CTA c owns TC blocks [c*T/G, (c+1)*T/G) (strict balance) or
// that range snapped to row-window starts (window mode). Windows cut by a
// CTA boundary write fp32 partial tiles to a workspace; k_reduce_partials
// sums them in CTA order, so results do not depend on timing.
//
// Pipeline. A ring of S stages, each holding P consecutive TC blocks of the
// CTA's range (barrier traffic is per stage, not per block).
//   warps 0-3   epilogue: tcgen05.ld 32x32b; each warp stages its 32 columns
//               x window rows of C in shared memory and issues one TMA tensor
//               store (plain per-lane stores stalled these warps and, through
//               the accumulator hand-off, the whole pipeline)
//   warps 4-5   UMMA issuers (one thread each; warp 4 also owns TMEM):
//               issuer m takes the stages s % 2 == m into its own set of
//               accumulators, so two MMA streams are in flight (a single
//               issuing thread cannot saturate the tensor pipe with these
//               small M128 x N16 x K8 instructions); the epilogue adds the
//               two partial accumulators in a fixed order
//   warps 6-9   loaders: cp.async 16-byte gathers of B rows (SparseAToX),
//               zero-fill for padded slots; stage s is owned by loader s % 4
//   warps 10-13 tile builders: zero + scatter TC-block values into A_b^T;
//               stage s is owned by tile builder s % 4; tile ids and values
//               of a stage are loaded one owned stage ahead
// Each warp owns a fixed residue class of stages, so it waits on every
// barrier phase of its stages in order (a parity wait more than one phase
// ahead would pass spuriously). Every wait is bounded (2 s) and records
// kErrWaitTimeout instead of hanging.
#include <cuda_bf16.h>
#include "spmm_sched.cuh"
#include "impl.h"

namespace dtc {
namespace {

constexpr int kEpiWarps = 4;
constexpr int kMmaWarp = 4;     // UMMA issuers: warps 4 and 5 (lane 0 each)
constexpr int kMmaWarps = 2;
constexpr int kLoadWarp0 = kMmaWarp + kMmaWarps;
constexpr int kLoadWarps = 4;
constexpr int kTileWarp0 = kLoadWarp0 + kLoadWarps;
constexpr int kTileWarps = 4;
constexpr int kThreads = 32 * (kTileWarp0 + kTileWarps);  // 448
constexpr int kXTileBytes = 4096;   // 8 rows x 128 fp32 features

// Byte offset, inside one 8-row x 128-feature fp32 tile, of 16-byte chunk
// `cc` (features 4cc..4cc+3) of row k, in the UMMA layout-type-1 atom order:
// atom = 32 features x 4 rows (512 B), 32-byte granule index XOR (row & 3).
__device__ __forceinline__ uint32_t x_offset_tf32(uint32_t k, uint32_t cc) {
  const uint32_t a = cc >> 3, j = cc & 7;
  const uint32_t g = (j >> 1) ^ (k & 3);
  return a * 1024 + (k >> 2) * 512 + (k & 3) * 128 + ((g << 1) | (j & 1)) * 16;
}

// WH = row-window height (the UMMA N dimension): 16 or 32.
template <int NT, int P, int S, int WH>
struct Cfg {
  static_assert(S % kLoadWarps == 0 && S % kTileWarps == 0 && S % kMmaWarps == 0,
                "stage ownership");
  static_assert(P * kBlkW <= 32, "one SparseAToX entry per lane");
  static_assert(WH == 16 || WH == 32, "window height");
  static constexpr int kNacc = (NT * WH > 64) ? 2 : 4;  // TMEM accumulator buffers in flight
  static constexpr int kYB = WH * kBlkW * 4;            // WH x 8 fp32, K-major core matrices
  static constexpr int kStageX = P * NT * kXTileBytes;
  static constexpr int kStageY = P * kYB;
  static constexpr int kX = S * kStageX;
  static constexpr int kY = S * kStageY;
  static constexpr int kStgW = WH * 32 * 4;               // one epilogue warp's C tile
  static constexpr int kStg = kEpiWarps * 2 * kStgW;       // double-buffered per warp
  static constexpr int kBars = (2 * S + 2 * kNacc) * 8;
  static constexpr int kSmem = kX + kY + kStg + kBars + 16 + 1024;  // + alignment slack
  static constexpr int kCols = kMmaWarps * kNacc * NT * WH;  // TMEM columns used
  static_assert(kCols <= 512, "TMEM budget");
  static constexpr uint32_t kTmemCols = kCols <= 32 ? 32 : kCols <= 64 ? 64 : kCols <= 128 ? 128
                                        : kCols <= 256 ? 256 : 512;
};

template <int NT, int P, int S, int WH>
__global__ void __launch_bounds__(kThreads, 1) k_spmm_tf32(const __grid_constant__ Params p) {
  using K = Cfg<NT, P, S, WH>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* xring = smem;
  uint8_t* yring = smem + K::kX;
  uint8_t* stg = yring + K::kY;          // [4 warps][2][WH x 32] fp32 C staging
  uint64_t* bars = (uint64_t*)(stg + K::kStg);
  uint64_t* full = bars;                 // [S] 32 cp.async arrivals + 1 tile arrival
  uint64_t* empty = bars + S;            // [S] UMMA commit
  uint64_t* acc_full = bars + 2 * S;     // [kNacc] UMMA commit
  uint64_t* acc_empty = acc_full + K::kNacc;  // [kNacc] 4 epilogue warps
  uint32_t* tmem_slot = (uint32_t*)(acc_empty + K::kNacc);
  volatile uint32_t* abort_flag = tmem_slot + 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x;
  const int col0 = blockIdx.y * NT * 128;      // this CTA's feature slice
  const int ncols = (p.N - col0) < NT * 128 ? (p.N - col0) : NT * 128;
  const int nck = ncols >> 2;                  // 16-byte chunks per gathered row

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&full[i], 32 + 1);
      mbar_init(&empty[i], 1);
    }
    for (int i = 0; i < K::kNacc; ++i) {
      mbar_init(&acc_full[i], kMmaWarps);
      mbar_init(&acc_empty[i], kEpiWarps);
    }
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (warp == kMmaWarp) {
    tmem_alloc(tmem_slot, K::kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  int64_t b0, b1;
  cta_range(p, c, b0, b1);
  const int64_t nblk = b1 - b0;
  const int64_t nstage = (nblk + P - 1) / P;

  if (warp >= kLoadWarp0 && warp < kLoadWarp0 + kLoadWarps) {
    // ------------------------------------------------------------ loaders
    const int lw = warp - kLoadWarp0;
    auto row_of = [&](int64_t st) -> int32_t {  // SparseAToX entry of this lane
      const int64_t b = b0 + st * P + (lane >> 3);
      return (lane < P * kBlkW && st < nstage && b < b1) ? __ldg(p.s2x + b * kBlkW + (lane & 7))
                                                         : 0;
    };
    __shared__ int32_t rows_sm[kLoadWarps][32];  // SparseAToX of the stage being loaded
    int32_t rows = row_of(lw);
    for (int64_t st = lw; st < nstage; st += kLoadWarps) {
      const int s = (int)(st % S);
      const uint32_t n = (uint32_t)(st / S);
      const int32_t nxt = row_of(st + kLoadWarps);  // prefetch this warp's next stage
      const bool got = mbar_wait(&empty[s], (n & 1) ^ 1, p.err);
      if (!__all_sync(0xffffffffu, got) || *abort_flag) { *abort_flag = 1; break; }
      const int64_t sb = b0 + st * P;
      const int nb = (int)((b1 - sb) < P ? (b1 - sb) : P);
      const uint32_t xs = smem_u32(xring + (size_t)s * K::kStageX);
      if (nck == NT * 32) {
        // full 128-feature tiles: one gathered row per warp instruction
        for (int pb = 0; pb < nb; ++pb) {
#pragma unroll
          for (int k = 0; k < kBlkW; ++k) {
            const int32_t r = __shfl_sync(0xffffffffu, rows, pb * kBlkW + k);
            const bool pad = (k > 0 && r == 0);  // unused slot (columns ascend in a block)
            const float* src = p.B + (int64_t)(pad ? 0 : r) * p.N + col0;
#pragma unroll
            for (int t = 0; t < NT; ++t)
              cp_async16(xs + (pb * NT + t) * kXTileBytes + x_offset_tf32(k, lane),
                         src + (t * 32 + lane) * 4, pad ? 0u : 16u);
          }
        }
      } else {
        // partial slice: lanes flattened over (gathered row, 16-byte chunk)
        rows_sm[lw][lane] = rows;
        __syncwarp();
        for (int idx = lane; idx < nb * kBlkW * nck; idx += 32) {
          const int rowi = idx / nck, cc = idx - rowi * nck;
          const int k = rowi & 7, pb = rowi >> 3;
          const int32_t r = rows_sm[lw][rowi];
          const bool pad = (k > 0 && r == 0);
          const float* src = p.B + (int64_t)(pad ? 0 : r) * p.N + col0;
          cp_async16(xs + (pb * NT + (cc >> 5)) * kXTileBytes + x_offset_tf32(k, cc & 31),
                     src + cc * 4, pad ? 0u : 16u);
        }
        __syncwarp();
      }
      cp_async_arrive_noinc(&full[s]);
      rows = nxt;
    }
  } else if (warp >= kTileWarp0) {
    // ------------------------------------------------------ tile builders
    const int tw = warp - kTileWarp0;
    auto offs_of = [&](int64_t st) -> int32_t {
      const int64_t sb = b0 + st * P;
      return (st < nstage && lane <= P && sb + lane <= b1) ? __ldg(p.toff + sb + lane) : 0;
    };
    // Tile ids and values of the first 64 entries of a stage are loaded one
    // owned stage ahead (offsets two ahead), so their global-load latency
    // overlaps the previous stage's work instead of stalling this one.
    int32_t offv = offs_of(tw);
    int32_t offn = offs_of(tw + kTileWarps);
    uint32_t pt0 = 0, pt1 = 0;
    float pv0 = 0.0f, pv1 = 0.0f;
    auto fetch = [&](int64_t st, int32_t ov) {
      const int64_t sb = b0 + st * P;
      const int nbx = st < nstage ? (int)((b1 - sb) < P ? (b1 - sb) : P) : 0;
      const int32_t f0 = __shfl_sync(0xffffffffu, ov, 0), f1 = __shfl_sync(0xffffffffu, ov, nbx);
      const int32_t e = f0 + lane;
      pt0 = (e < f1) ? __ldg(p.tile + e) : 0u;
      pv0 = (e < f1) ? (p.vals ? __ldg(p.vals + e) : 1.0f) : 0.0f;
      pt1 = (e + 32 < f1) ? __ldg(p.tile + e + 32) : 0u;
      pv1 = (e + 32 < f1) ? (p.vals ? __ldg(p.vals + e + 32) : 1.0f) : 0.0f;
    };
    fetch(tw, offv);
    for (int64_t st = tw; st < nstage; st += kTileWarps) {
      const int s = (int)(st % S);
      const uint32_t n = (uint32_t)(st / S);
      const int32_t nxt = offs_of(st + 2 * kTileWarps);
      const uint32_t ct0 = pt0, ct1 = pt1;
      const float cv0 = pv0, cv1 = pv1;
      fetch(st + kTileWarps, offn);
      const int64_t sb = b0 + st * P;
      const int nb = (int)((b1 - sb) < P ? (b1 - sb) : P);
      int32_t off[P + 1];
#pragma unroll
      for (int k = 0; k <= P; ++k) off[k] = __shfl_sync(0xffffffffu, offv, k);
      const bool got = mbar_wait(&empty[s], (n & 1) ^ 1, p.err);
      if (!__all_sync(0xffffffffu, got) || *abort_flag) { *abort_flag = 1; break; }
      uint8_t* ys = yring + (size_t)s * K::kStageY;
#pragma unroll
      for (int z = lane; z < P * K::kYB / 16; z += 32)
        reinterpret_cast<float4*>(ys)[z] = make_float4(0.f, 0.f, 0.f, 0.f);
      __syncwarp();
      const int32_t e0 = off[0], e1 = off[nb];
      for (int32_t e = e0 + lane; e < e1; e += 32) {
        int pb = 0;
#pragma unroll
        for (int q = 1; q < P; ++q) pb += (q < nb && e >= off[q]) ? 1 : 0;
        const int32_t i = (e - e0) >> 5;  // chunk of this entry
        const uint32_t pos = i == 0 ? ct0 : i == 1 ? ct1 : __ldg(p.tile + e);
        const float v = i == 0 ? cv0 : i == 1 ? cv1 : (p.vals ? __ldg(p.vals + e) : 1.0f);
        if (pos < WH * kBlkW) {
          if (v != 0.0f) {
            uint32_t t32;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t32) : "f"(v));
            *reinterpret_cast<uint32_t*>(ys + pb * K::kYB + y_offset(pos)) = t32;
          }
        } else {
          atomicOr(p.err, kErrBadIndex);
        }
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&full[s]);
      offv = offn;
      offn = nxt;
    }
  } else if (warp >= kMmaWarp && warp < kMmaWarp + kMmaWarps) {
    // ------------------------------------------------------------- UMMA
    if (lane == 0) {
      const int m = warp - kMmaWarp;  // this issuer's stages: st % kMmaWarps == m
      int32_t ws, we;
      cta_windows(p, c, b0, b1, ws, we);
      constexpr uint32_t idesc = umma_idesc(2, 128, WH, 1, 0);
      // Descriptors advance by adding (byte offset >> 4) to the start-address
      // field (shared addresses < 256 KB fit its 14 bits, no carry out).
      const uint64_t adesc0 = umma_desc(smem_u32(xring), 1024, 512, 1);
      const uint64_t bdesc0 = umma_desc(smem_u32(yring), 128, 256, 0);
      uint32_t q = 0;        // segment counter
      bool ok = true;
      int64_t r0 = ws < we ? __ldg(p.rwo + ws) : 0;
      int64_t r1 = ws < we ? __ldg(p.rwo + ws + 1) : 0;
      for (int32_t w = ws; w < we && ok; ++w) {
        const int64_t r2 = (w + 2 <= p.nwin) ? __ldg(p.rwo + w + 2) : 0;  // next window's end
        const int64_t s0 = r0 > b0 ? r0 : b0, s1 = r1 < b1 ? r1 : b1;
        r0 = r1;
        r1 = r2;
        if (s0 >= s1) continue;  // empty window, or no blocks of it in this range
        const int a = (int)(q % K::kNacc);
        if (!mbar_wait(&acc_empty[a], ((q / K::kNacc) & 1) ^ 1, p.err)) { ok = false; break; }
        tc_fence_after();
        const uint32_t dtm = tmem_base + (uint32_t)((m * K::kNacc + a) * NT * WH);
        uint32_t acc = 0;
        // this issuer's stages that intersect [s0, s1)
        int64_t st = (s0 - b0) / P;
        st += (m - (int)(st % kMmaWarps) + kMmaWarps) % kMmaWarps;
        const int64_t st_last = (s1 - 1 - b0) / P;
        for (; st <= st_last; st += kMmaWarps) {
          const int s = (int)(st % S);
          const int64_t sb = b0 + st * P;                 // first block of stage st
          const int64_t lo = sb > s0 ? sb : s0;
          const int64_t hi = (sb + P) < s1 ? (sb + P) : s1;
          if (lo == sb) {  // first visit of this stage (segments are walked in order)
            if (!mbar_wait(&full[s], (uint32_t)(st / S) & 1, p.err)) { ok = false; break; }
            fence_proxy_async_smem();  // cp.async (generic proxy) data -> UMMA reads
            tc_fence_after();
          }
          uint64_t bdesc = bdesc0 + (uint64_t)((s * K::kStageY + (int)(lo - sb) * K::kYB) >> 4);
          uint64_t adesc =
              adesc0 + (uint64_t)((s * K::kStageX + (int)(lo - sb) * NT * kXTileBytes) >> 4);
          for (int64_t b = lo; b < hi; ++b) {
#pragma unroll
            for (int t = 0; t < NT; ++t)
              mma_tf32(dtm + t * WH, adesc + (uint64_t)(t * (kXTileBytes >> 4)), bdesc, idesc, acc);
            acc = 1;
            adesc += (uint64_t)((NT * kXTileBytes) >> 4);
            bdesc += (uint64_t)(K::kYB >> 4);
          }
          if (hi == sb + P || hi == b1) tc_commit(&empty[s]);  // stage fully consumed
        }
        if (!ok) break;
        tc_commit(&acc_full[a]);  // also when this issuer had no block in the segment
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
    uint32_t su = 0;      // C tiles this warp has staged (selects the staging buffer)
    int64_t rn0 = ws < we ? __ldg(p.rwo + ws) : 0;
    int64_t rn1 = ws < we ? __ldg(p.rwo + ws + 1) : 0;
    for (int32_t w = ws; w < we; ++w) {
      const int64_t r0 = rn0, r1 = rn1;
      rn0 = rn1;
      rn1 = (w + 2 <= p.nwin) ? __ldg(p.rwo + w + 2) : 0;  // prefetch the next window's end
      const int64_t row0 = (int64_t)w * WH;
      if (r0 == r1) {  // empty window: C rows are zero
        for (int f = col0 + ew * 32 + lane; f < col0 + ncols; f += 128)
          for (int r = 0; r < WH && row0 + r < p.M; ++r)
            p.C[(row0 + r) * p.N + f] = epilogue(p, 0.0f, f);
        continue;
      }
      if ((r0 > b0 ? r0 : b0) >= (r1 < b1 ? r1 : b1)) continue;
      const int a = (int)(q % K::kNacc);
      const bool got = mbar_wait(&acc_full[a], (q / K::kNacc) & 1, p.err);
      if (!__all_sync(0xffffffffu, got)) { *abort_flag = 1; break; }
      tc_fence_after();
      float* out;
      bool guard_rows = true;
      if (p.mode == 1 && (r0 < b0 || r1 > b1)) {  // window cut by a CTA boundary
        const int slot = (r0 < b0) ? 2 * c : 2 * c + 1;
        out = p.part + (size_t)slot * WH * p.N;
        guard_rows = false;
      } else {
        out = p.C + row0 * p.N;
      }
      // issuers that hold part of this segment: stages of [s0, s1) mod kMmaWarps
      const int64_t s0 = r0 > b0 ? r0 : b0, s1 = r1 < b1 ? r1 : b1;
      const int64_t st0 = (s0 - b0) / P, st1 = (s1 - 1 - b0) / P;
      const bool both = st1 > st0;
      const int m0 = (int)(st0 % kMmaWarps);
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        uint32_t v[WH / 16][16], u[WH / 16][16];
        const uint32_t lane_addr = tmem_base + ((uint32_t)(ew * 32) << 16);
        const uint32_t c0 = (uint32_t)(((m0 * K::kNacc + a) * NT + t) * WH);
        const uint32_t c1 = (uint32_t)((((1 - m0) * K::kNacc + a) * NT + t) * WH);
#pragma unroll
        for (int h = 0; h < WH / 16; ++h) {
          tmem_ld16(lane_addr + c0 + h * 16, v[h]);
          if (both) tmem_ld16(lane_addr + c1 + h * 16, u[h]);
        }
        tmem_ld_wait();
        float x[WH];
        if (both) {  // fixed order: issuer 0's partial + issuer 1's partial
#pragma unroll
          for (int r = 0; r < WH; ++r) {
            const float pv = __uint_as_float(v[r >> 4][r & 15]);
            const float pu = __uint_as_float(u[r >> 4][r & 15]);
            x[r] = m0 == 0 ? pv + pu : pu + pv;
          }
        } else {
#pragma unroll
          for (int r = 0; r < WH; ++r) x[r] = __uint_as_float(v[r >> 4][r & 15]);
        }
        const int f = col0 + t * 128 + ew * 32 + lane;
        if (t == NT - 1) {
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&acc_empty[a]);
        }
        if (!guard_rows) {  // partial tile of a cut window: raw sums to the workspace
          if (f < p.N) {
#pragma unroll
            for (int r = 0; r < WH; ++r) out[r * p.N + f] = x[r];
          }
        } else if (col0 + t * 128 + ew * 32 < p.N) {
          // finished tile: this warp's 32 columns x WH rows go through shared
          // memory to one TMA store (rows past M and columns past N are clipped
          // by the tensor map); the other buffer's store may still be reading
          float* sb = reinterpret_cast<float*>(stg + (ew * 2 + (su & 1)) * K::kStgW);
          __syncwarp();  // lane 0 has waited for this buffer's previous store
#pragma unroll
          for (int r = 0; r < WH; ++r) sb[r * 32 + lane] = epilogue(p, x[r], f < p.N ? f : 0);
          fence_proxy_async_smem();
          __syncwarp();
          if (lane == 0) {
            tma_store_2d(&p.cmap, sb, col0 + t * 128 + ew * 32, (int32_t)row0);
            bulk_commit();
            bulk_wait_read<1>();
          }
          ++su;
        }
      }
      ++q;
    }
    if (lane == 0) bulk_wait_all();
  }

  tc_fence_before();
  __syncthreads();
  if (warp == kMmaWarp) {
    tc_fence_after();
    tmem_dealloc(tmem_base, K::kTmemCols);
  }
}

// rwo[w] = first block of window w, from the sorted window id of every block.
// Ids come from the caller: an id outside [0, nwin) or a descending pair is
// reported through kErrBadIndex, and the written range is clamped to the
// (nwin + 1)-entry table, so a bad id never writes outside it.
__global__ void k_rowid_to_rwo(const int32_t* __restrict__ rowid, int64_t T, int32_t nwin,
                               int32_t* __restrict__ rwo, uint32_t* err) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b <= T; b += stride) {
    const int32_t prev = (b == 0) ? -1 : __ldg(rowid + b - 1);
    const int32_t cur = (b == T) ? nwin : __ldg(rowid + b);
    const bool bad = (b < T && (cur < 0 || cur >= nwin)) || cur < prev;
    if (bad) atomicOr(err, kErrBadIndex);
    const int32_t lo = prev < -1 ? -1 : (prev > nwin ? nwin : prev);
    const int32_t hi = cur < -1 ? -1 : (cur > nwin ? nwin : cur);
    for (int32_t w = lo + 1; w <= hi; ++w) rwo[w] = (int32_t)b;
  }
}

template <int NT, int P, int S, int WH>
dtc_status launch_tf32(const Params& p, int slices, cudaStream_t st) {
  constexpr int smem = Cfg<NT, P, S, WH>::kSmem;
  static_assert(smem <= 227 * 1024, "shared memory budget");
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    DTC_CUDA(cudaFuncSetAttribute(k_spmm_tf32<NT, P, S, WH>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr_set[dev & 63] = true;
  }
  dim3 grid((unsigned)p.G, (unsigned)slices);
  k_spmm_tf32<NT, P, S, WH><<<grid, kThreads, smem, st>>>(p);
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
                          float* part, cudaStream_t st, int ntile, Epilogue epi, int H) {
  DTC_REQUIRE(M >= 0 && N >= 1 && T >= 0, "bad sizes");
  DTC_REQUIRE(N % 4 == 0, "tcgen05 path needs N % 4 == 0 (16-byte row segments)");
  DTC_REQUIRE(((uintptr_t)B & 15) == 0, "B must be 16-byte aligned");
  DTC_REQUIRE(H == 16 || H == 32, "window height must be 16 or 32");
  DTC_REQUIRE(nwin == (M + H - 1) / H, "num_windows must be ceil(num_nodes / window height)");
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
  p.rwo = rwo; p.tile = tile; p.toff = toff; p.s2x = s2x; p.vals = vals; p.B = B;
  p.C = C; p.part = part; p.err = device_error_word();
  p.bias = epi.bias; p.relu = epi.relu;
  p.M = M; p.nwin = nwin; p.N = N; p.T = T; p.mode = mode; p.H = H;
  DTC_REQUIRE(((uintptr_t)C & 15) == 0, "C must be 16-byte aligned");
  dtc_status es = encode_c_map(&p.cmap, C, M, N, H);
  if (es != DTC_OK) return es;
  int G = grid > 0 ? grid : default_grid();
  if ((int64_t)G > T) G = (int)T;
  p.G = G;
  // N-tiles (128 features each) per CTA: all of N up to 4 tiles unless capped
  // by `ntile`; wider slices of N go to more CTAs (grid.y).
  int nt = N <= 128 ? 1 : N <= 256 ? 2 : 4;
  if (ntile == 1 || ntile == 2) nt = nt < ntile ? nt : ntile;
  if (H == 32) {
    if (nt == 1) return launch_tf32<1, 4, 8, 32>(p, (N + 127) / 128, st);
    if (nt == 2) return launch_tf32<2, 2, 8, 32>(p, (N + 255) / 256, st);
    return launch_tf32<4, 1, 8, 32>(p, (N + 511) / 512, st);
  }
  if (nt == 1) return launch_tf32<1, 4, 8, 16>(p, (N + 127) / 128, st);
  if (nt == 2) return launch_tf32<2, 2, 8, 16>(p, (N + 255) / 256, st);
  return launch_tf32<4, 1, 8, 16>(p, (N + 511) / 512, st);
}

size_t spmm_partials_bytes(int64_t T, int32_t N, int grid, int H) {
  int G = grid > 0 ? grid : default_grid();
  if ((int64_t)G > T) G = (int)(T > 0 ? T : 1);
  return (size_t)2 * G * H * (size_t)N * sizeof(float);
}

dtc_status rowid_to_rwo(const int32_t* rowid, int64_t T, int32_t nwin, int32_t* rwo,
                        cudaStream_t st) {
  int64_t n = T + 1;
  unsigned g = (unsigned)((n + 255) / 256);
  if (g > 65535u * 16) g = 65535u * 16;
  k_rowid_to_rwo<<<g, 256, 0, st>>>(rowid, T, nwin, rwo, device_error_word());
  DTC_CUDA(cudaGetLastError());
  return DTC_OK;
}

}  // namespace dtc
