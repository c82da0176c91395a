// Split-precision TC-block SpMM: bf16 operands on tcgen05 kind::f16 with
// fp32 accumulation in TMEM, B gathered from a compact storage form.
//
// Forms (B storage, see formats.cu):
//   SPLIT24 : bf16 hi plane + u8 extension plane (3 bytes/element). The
//             tile warps rebuild lo = b24 - hi (exact in bf16) in shared
//             memory, so B_hi + B_lo reproduces B rounded to 16 significant
//             bits.
//   BF16    : bf16 plane (2 bytes/element); lo = 0.
//   FP8     : e4m3 plane + fp32 row scale (1 byte/element); the tile warps
//             expand q * scale[row] to bf16 hi; lo = 0.
//   BF16X2  : bf16 hi plane + bf16 lo plane (4 bytes/element, the fp32 byte
//             count): the loaders copy both planes straight into the operand
//             tile, no rebuild on the CUDA cores.
// A values are split the same way: A_hi = bf16(a), A_lo = bf16(a - A_hi).
//
// One UMMA per TC block and 128-feature tile computes every product term:
//   UMMA A operand (M = 128 features x K = 16): rows k < 8 are B_hi of the
//   block's 8 gathered rows, rows k >= 8 are B_lo (MN-major, 128-byte swizzle)
//   UMMA B operand (K = 16 x N = 32, K-major): columns 0..15 hold A_hi^T
//   (over both K halves), columns 16..31 hold A_lo^T (over the hi half; over
//   the lo half too for the 4-term form).
//   D[:, r] + D[:, 16 + r] = (B_hi + B_lo) A_hi^T + (B_hi [+ B_lo]) A_lo^T.
// The N = 32 instruction costs the same tensor-pipe time as N = 16, so the
// full product takes one instruction per block, like the tf32 form, while
// gathering 3 (SPLIT24), 2 (BF16), 1 (FP8) or 4 (BF16X2) bytes per element.
//
// Schedule, work split, producer warp and the deterministic reduction are the
// tf32 kernel's (spmm_tc.cu, spmm_sched.cuh). Warp roles: epilogue 0-3, UMMA
// issuers 4-5, loaders 6-9 (cp.async of the planes), tile builders 10-13
// (A_hi / A_lo tiles), producer 14, and for the forms that rebuild operand
// rows on the CUDA cores (SPLIT24, FP8) converters 15-22, which wait for a
// stage's gathered rows and rebuild the bf16 operand rows in place (480 or
// 736 threads). A stage is released to the UMMA issuers by the loader's
// cp.async arrivals and the tile builder (BF16, BF16X2), or by the tile
// builder and the converter. Finished C tiles leave through shared memory and
// per-warp TMA tensor stores (16 rows x 32 columns). At window height 32 with
// one N-tile, the forms that stage a second plane (SPLIT24, FP8) hold 3
// blocks per stage so the 32-row A tiles and the staging fit in shared memory.
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include "spmm_sched.cuh"
#include "impl.h"

namespace dtc {
namespace {

constexpr int kEpiWarps = 4;     // warps 0-3
constexpr int kMmaWarp = 4;      // warps 4-5
constexpr int kMmaWarps = 2;
constexpr int kLoadWarp0 = kMmaWarp + kMmaWarps;   // warps 6-9
constexpr int kLoadWarps = 4;
constexpr int kTileWarp0 = kLoadWarp0 + kLoadWarps;  // warps 10-13
constexpr int kTileWarps = 4;
constexpr int kProdWarp = kTileWarp0 + kTileWarps;   // warp 14
constexpr int kConvWarp0 = kProdWarp + 1;            // warps 15-22 (SPLIT24, FP8)
constexpr int kConvWarps = 8;
constexpr int kTileBytes = 4096;  // per block and 128-feature tile: 16 K rows x 128 bf16

enum { kFormSplit24 = 0, kFormBF16 = 1, kFormFP8 = 2, kFormBF16X2 = 3 };

// WH = row-window height; the UMMA N dimension is 2 WH (A_hi^T | A_lo^T).
// BW = TC-block width (8 or 16): a block of width 16 is two 8-slot halves,
// each one K = 16 (hi | lo) MMA into the same accumulator.
template <int FORM, int NT, int P, int S, int WH, int BW>
struct SCfg {
  static constexpr bool kConv = (FORM == kFormSplit24 || FORM == kFormFP8);
  static constexpr int kThreads = 32 * (kConvWarp0 + (kConv ? kConvWarps : 0));
  static_assert(S % kLoadWarps == 0 && S % kTileWarps == 0 && S % kConvWarps == 0, "ownership");
  static_assert((S & (S - 1)) == 0 && S % 2 == 0, "stage counters are kept modulo 2^32");
  static_assert(kConvWarps <= kEndStages, "end markers");
  static_assert(BW == 8 || BW == 16, "block width");
  static_assert(P * BW <= 32, "one SparseAToX entry per lane");
  static_assert(WH * BW <= 256, "tile ids are bytes");
  static_assert(WH == 16 || WH == 32, "window height");
  static_assert(NT * WH <= 64, "TMEM budget: two accumulator sets per issuer");
  static constexpr int kAccCols = NT * 2 * WH;  // TMEM columns of one accumulator set
  static constexpr int kNacc = 512 / (kMmaWarps * kAccCols) < 4 ? 512 / (kMmaWarps * kAccCols) : 4;
  static constexpr int kSub = BW / 8;  // 8-slot halves per block
  static constexpr int kYB8 = 64 * WH;  // 16 K x 2WH N bf16, K-major core matrices
  static constexpr int kYB = kSub * kYB8;  // one block's A^T tile
  static constexpr int kStageX = P * NT * kSub * kTileBytes;
  static constexpr int kRowStage = NT * 128;  // staged bytes of one gathered row (u8 / e4m3)
  static constexpr int kStageE = kConv ? P * BW * kRowStage : 0;
  static constexpr int kStageY = P * kYB;
  static constexpr int kX = S * kStageX;
  static constexpr int kE = S * kStageE;
  static constexpr int kY = S * kStageY;
  static constexpr int kBars = (3 * S + 2 * kNacc + kMmaWarps) * 8;
  static constexpr int kStgW = 16 * 32 * 4;          // one epilogue warp's 16-row C tile
  static constexpr int kStg = kEpiWarps * 2 * kStgW;  // double-buffered per warp
  static constexpr int kSmem = kX + kE + kY + kStg + kSchedBytes + kBars + 16 + 1024;
  static_assert(kSmem <= 232448, "dynamic shared memory per CTA");
  static constexpr int kCols = kMmaWarps * kNacc * kAccCols;
  static_assert(kCols <= 512, "TMEM budget");
  static constexpr uint32_t kTmemCols = kCols <= 32 ? 32 : kCols <= 64 ? 64 : kCols <= 128 ? 128
                                        : kCols <= 256 ? 256 : 512;
};

// Byte offset in one block tile of the 16-byte chunk j (features 8j..8j+7)
// of K row k16 (0..7 hi, 8..15 lo): bf16 MN-major, 128-byte swizzle with
// 16-byte granules; atoms of 64 features x 8 rows (LBO = 1024 B between the
// two feature atoms, SBO = 2048 B between the hi and lo row groups).
__device__ __forceinline__ uint32_t x_offset_bf16(uint32_t k16, uint32_t j) {
  const uint32_t kk = k16 & 7;
  return (k16 >> 3) * 2048 + (j >> 3) * 1024 + kk * 128 + (((j & 7) ^ kk) << 4);
}

// Byte offset of B-operand element (n, k): K-major, no swizzle, LBO = 128 B
// between K halves, SBO = 256 B between 8-column groups.
__device__ __forceinline__ uint32_t ysplit_offset(uint32_t n, uint32_t k) {
  return (n & 7) * 16 + (n >> 3) * 256 + (k >> 3) * 128 + (k & 7) * 2;
}

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  return __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

template <int FORM, int NT, int P, int S, bool FOUR, int WH, int BW>
__global__ void __launch_bounds__(SCfg<FORM, NT, P, S, WH, BW>::kThreads, 1)
    k_spmm_split(const __grid_constant__ Params p) {
  using K = SCfg<FORM, NT, P, S, WH, BW>;
  const uint64_t t_entry = global_timer_ns();
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* xring = smem;
  uint8_t* ering = smem + K::kX;
  uint8_t* yring = ering + K::kE;
  uint8_t* stg = yring + K::kY;  // [4 warps][2][16 x 32] fp32 C staging
  const SchedRings rings = carve_rings(stg + K::kStg);
  uint64_t* bars = (uint64_t*)(stg + K::kStg + kSchedBytes);
  uint64_t* loaded = bars;               // [S] 32 cp.async arrivals (converter forms)
  uint64_t* full = bars + S;             // [S] see the header comment
  uint64_t* empty = bars + 2 * S;        // [S] the owning issuer's UMMA commit
  uint64_t* acc_full = bars + 3 * S;     // [kNacc] one commit per issuer
  uint64_t* acc_empty = acc_full + K::kNacc;
  uint64_t* drain = acc_empty + K::kNacc;     // [kMmaWarps] an issuer's last commit
  uint32_t* tmem_slot = (uint32_t*)(drain + kMmaWarps);
  volatile uint32_t* abort_flag = tmem_slot + 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int col0 = blockIdx.y * NT * 128;
  const int ncols = (p.N - col0) < NT * 128 ? (p.N - col0) : NT * 128;

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&loaded[i], 32);
      mbar_init(&full[i], K::kConv ? 2 : 32 + 1);
      mbar_init(&empty[i], 1);  // the owning issuer's MMA commit
    }
    for (int i = 0; i < K::kNacc; ++i) {
      mbar_init(&acc_full[i], kMmaWarps);
      mbar_init(&acc_empty[i], kEpiWarps);
    }
    for (int i = 0; i < kMmaWarps; ++i) mbar_init(&drain[i], 1);
    // metadata: loader + tile builder (+ converter); records: every epilogue
    // warp and issuer
    init_rings(rings, K::kConv ? 3 : 2, kEpiWarps + kMmaWarps);
    *abort_flag = 0;
    fence_mbar_init();
  }
  if (FORM == kFormBF16 || FORM == kFormFP8) {  // lo rows stay zero for one-plane forms
    for (int i = threadIdx.x; i < S * P * NT * K::kSub; i += blockDim.x) {  // every block tile
      float4* lo = reinterpret_cast<float4*>(xring + (size_t)i * kTileBytes + 2048);
      for (int z = 0; z < 2048 / 16; ++z) lo[z] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    fence_proxy_async_smem();
  }
  if (warp == kMmaWarp) {
    tmem_alloc(tmem_slot, K::kTmemCols);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_slot;

  if (warp == kProdWarp) {
    produce<P, BW, kMmaWarps>(p, rings, lane, abort_flag);
  } else if (warp >= kLoadWarp0 && warp < kLoadWarp0 + kLoadWarps) {
    // ------------------------------------------------------------ loaders
    const int lw = warp - kLoadWarp0;
    __shared__ int32_t rows_sm[kLoadWarps][32];  // SparseAToX of the stage being loaded
    const uint8_t* plane0 = reinterpret_cast<const uint8_t*>(p.B);
    const uint8_t* plane1 = reinterpret_cast<const uint8_t*>(p.B1);
    for (int64_t st = lw;; st += kLoadWarps) {
      const int ms = (int)(st % kMetaDepth);
      if (!warp_wait(&rings.meta_full[ms], (uint32_t)(st / kMetaDepth) & 1, p.err, abort_flag))
        break;
      const int nb = rings.meta[ms].nb;
      const int32_t rows = rings.meta[ms].s2x[lane];
      __syncwarp();
      if (lane == 0) mbar_arrive(&rings.meta_empty[ms]);
      if (nb < 0) break;
      const int s = (int)(st % S);
      const uint32_t n = (uint32_t)(st / S);
      if (!warp_wait(&empty[s], (n & 1) ^ 1, p.err, abort_flag)) break;
      const uint32_t xs = smem_u32(xring + (size_t)s * K::kStageX);
      const uint32_t es = smem_u32(ering + (size_t)s * K::kStageE);
      const uint8_t* eplane = FORM == kFormSplit24 ? plane1 : plane0;
      if (ncols == NT * 128) {
        // full 128-feature tiles: RPI gathered rows per warp instruction,
        // CPR 16-byte chunks per row (compile-time)
        for (int pb = 0; pb < nb; ++pb) {
          if (FORM != kFormFP8) {  // bf16 hi (+ lo) plane -> K rows of the block tile, swizzled
            constexpr int CPR = NT * 16, RPI = CPR >= 32 ? 1 : 32 / CPR;
            constexpr int IPR = CPR >= 32 ? CPR / 32 : 1;
            constexpr int NPL = FORM == kFormBF16X2 ? 2 : 1;  // plane pl -> K rows 8 pl .. 8 pl + 7
#pragma unroll
            for (int pl = 0; pl < NPL; ++pl) {
              const uint8_t* base = pl ? plane1 : plane0;
#pragma unroll
              for (int k0 = 0; k0 < BW; k0 += RPI) {
                const int k = k0 + (RPI > 1 ? lane / CPR : 0);
                const int32_t r = __shfl_sync(0xffffffffu, rows, pb * BW + k);
                const bool pad = (k > 0 && r == 0);  // unused slot (columns ascend in a block)
                const uint8_t* src = base + ((int64_t)(pad ? 0 : r) * p.N + col0) * 2;
#pragma unroll
                for (int ii = 0; ii < IPR; ++ii) {
                  const int cc = (RPI > 1 ? lane % CPR : lane) + ii * 32;
                  cp_async16(xs + ((pb * NT + (cc >> 4)) * K::kSub + (k >> 3)) * kTileBytes +
                                 x_offset_bf16(pl * 8 + (k & 7), cc & 15),
                             src + cc * 16, pad ? 0u : 16u);
                }
              }
            }
          }
          if (K::kConv) {  // u8 ext / e4m3 plane -> staging
            constexpr int CPR = NT * 8, RPI = CPR >= 32 ? 1 : 32 / CPR;
            constexpr int IPR = CPR >= 32 ? CPR / 32 : 1;
#pragma unroll
            for (int k0 = 0; k0 < BW; k0 += RPI) {
              const int k = k0 + (RPI > 1 ? lane / CPR : 0);
              const int32_t r = __shfl_sync(0xffffffffu, rows, pb * BW + k);
              const bool pad = (k > 0 && r == 0);
              const uint8_t* src = eplane + (int64_t)(pad ? 0 : r) * p.N + col0;
#pragma unroll
              for (int ii = 0; ii < IPR; ++ii) {
                const int cc = (RPI > 1 ? lane % CPR : lane) + ii * 32;
                cp_async16(es + (pb * BW + k) * K::kRowStage + cc * 16, src + cc * 16,
                           pad ? 0u : 16u);
              }
            }
          }
        }
      } else {
        // partial slice: lanes flattened over (gathered row, 16-byte chunk)
        rows_sm[lw][lane] = rows;
        __syncwarp();
        const int nrow = nb * BW;
        if (FORM != kFormFP8) {
          const int nck = ncols >> 3;
          constexpr int NPL = FORM == kFormBF16X2 ? 2 : 1;
          for (int idx = lane; idx < NPL * nrow * nck; idx += 32) {
            const int pl = idx / (nrow * nck), id2 = idx - pl * nrow * nck;
            const int rowi = id2 / nck, cc = id2 - rowi * nck;
            const int k = rowi % BW, pb = rowi / BW;
            const int32_t r = rows_sm[lw][rowi];
            const bool pad = (k > 0 && r == 0);
            const uint8_t* src = (pl ? plane1 : plane0) + ((int64_t)(pad ? 0 : r) * p.N + col0) * 2;
            cp_async16(xs + ((pb * NT + (cc >> 4)) * K::kSub + (k >> 3)) * kTileBytes +
                           x_offset_bf16(pl * 8 + (k & 7), cc & 15),
                       src + cc * 16, pad ? 0u : 16u);
          }
        }
        if (K::kConv) {
          const int nck = ncols >> 4;
          for (int idx = lane; idx < nrow * nck; idx += 32) {
            const int rowi = idx / nck, cc = idx - rowi * nck;
            const int32_t r = rows_sm[lw][rowi];
            const bool pad = ((rowi % BW) > 0 && r == 0);
            const uint8_t* src = eplane + (int64_t)(pad ? 0 : r) * p.N + col0;
            cp_async16(es + rowi * K::kRowStage + cc * 16, src + cc * 16, pad ? 0u : 16u);
          }
        }
        __syncwarp();
      }
      cp_async_arrive_noinc(K::kConv ? &loaded[s] : &full[s]);
    }
    cp_async_wait_all();
  } else if (warp >= kTileWarp0 && warp < kTileWarp0 + kTileWarps) {
    // ------------------------------------------------------ tile builders
    const int tw = warp - kTileWarp0;
    // One stage's prefetched inputs: its offsets (lane k holds
    // TCblockoffset[sb + k]), block count (-1: end of work, -2: not fetched
    // yet), and the tile ids / values of its first 64 entries.
    struct Pf {
      int32_t offv;
      int nb;
      uint32_t t0, t1;
      float v0, v1;
    };
    bool ok = true;
    // Stages ahead of the one being built are only probed, never waited for:
    // the producer emits a stage's metadata after the window records of the
    // stages before it, and those records may need this warp's current stage
    // finished first.
    auto fetch = [&](int64_t st, Pf& f, bool wait) {
      f.nb = -2;
      f.offv = 0;
      f.t0 = f.t1 = 0;
      f.v0 = f.v1 = 0.0f;
      const int ms = (int)(st % kMetaDepth);
      const uint32_t par = (uint32_t)(st / kMetaDepth) & 1;
      if (!wait) {
        if (!__all_sync(0xffffffffu, mbar_try_wait(&rings.meta_full[ms], par))) return;
      } else if (!warp_wait(&rings.meta_full[ms], par, p.err, abort_flag)) {
        ok = false;
        return;
      }
      f.nb = rings.meta[ms].nb;
      f.offv = (f.nb >= 0 && lane <= f.nb) ? rings.meta[ms].toff[lane] : 0;
      __syncwarp();
      if (lane == 0) mbar_arrive(&rings.meta_empty[ms]);
      if (f.nb < 0) return;
      const int32_t f0 = __shfl_sync(0xffffffffu, f.offv, 0);
      const int32_t f1 = __shfl_sync(0xffffffffu, f.offv, f.nb);
      const int32_t e = f0 + lane;
      f.t0 = (e < f1) ? __ldg(p.tile + e) : 0u;
      f.v0 = (e < f1) ? (p.vals ? __ldg(p.vals + e) : 1.0f) : 0.0f;
      f.t1 = (e + 32 < f1) ? __ldg(p.tile + e + 32) : 0u;
      f.v1 = (e + 32 < f1) ? (p.vals ? __ldg(p.vals + e + 32) : 1.0f) : 0.0f;
    };
    Pf cur, n1, n2;
    fetch(tw, cur, true);
    if (ok && cur.nb >= 0) fetch(tw + kTileWarps, n1, false); else n1.nb = -1;
    for (int64_t st = tw; ok && cur.nb >= 0; st += kTileWarps) {
      // probe two stages ahead unless the next one is known to end the work
      // (an unprobed next stage, nb == -2, still lets this one be probed)
      if (n1.nb != -1) fetch(st + 2 * kTileWarps, n2, false); else n2.nb = -1;
      const int s = (int)(st % S);
      const uint32_t n = (uint32_t)(st / S);
      const int nb = cur.nb;
      int32_t off[P + 1];
#pragma unroll
      for (int k = 0; k <= P; ++k) off[k] = __shfl_sync(0xffffffffu, cur.offv, k);
      if (!warp_wait(&empty[s], (n & 1) ^ 1, p.err, abort_flag)) break;
      uint8_t* ys = yring + (size_t)s * K::kStageY;
      for (int z = lane; z < P * K::kYB / 16; z += 32)
        reinterpret_cast<float4*>(ys)[z] = make_float4(0.f, 0.f, 0.f, 0.f);
      __syncwarp();
      const int32_t e0 = off[0], e1 = off[nb];
      for (int32_t e = e0 + lane; e < e1; e += 32) {
        int pb = 0;
#pragma unroll
        for (int q = 1; q < P; ++q) pb += (q < nb && e >= off[q]) ? 1 : 0;
        const int32_t i = (e - e0) >> 5;  // chunk of this entry
        const uint32_t pos = i == 0 ? cur.t0 : i == 1 ? cur.t1 : __ldg(p.tile + e);
        const float v = i == 0 ? cur.v0 : i == 1 ? cur.v1 : (p.vals ? __ldg(p.vals + e) : 1.0f);
        if (pos >= WH * BW) {
          atomicOr(p.err, kErrBadIndex);
          continue;
        }
        if (v == 0.0f) continue;
        const uint32_t r = pos / BW, sfull = pos % BW, sl = sfull & 7;
        const __nv_bfloat16 hi = __float2bfloat16_rn(v);
        const uint16_t hb = __bfloat16_as_ushort(hi);
        const uint16_t lb = bf16_bits(v - __bfloat162float(hi));
        uint8_t* yb = ys + pb * K::kYB + (sfull >> 3) * K::kYB8;
        *reinterpret_cast<uint16_t*>(yb + ysplit_offset(r, sl)) = hb;
        *reinterpret_cast<uint16_t*>(yb + ysplit_offset(r, 8 + sl)) = hb;
        *reinterpret_cast<uint16_t*>(yb + ysplit_offset(WH + r, sl)) = lb;
        if (FOUR) *reinterpret_cast<uint16_t*>(yb + ysplit_offset(WH + r, 8 + sl)) = lb;
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&full[s]);
      cur = n1;
      n1 = n2;
      if (cur.nb == -2) fetch(st + kTileWarps, cur, true);  // not ready when probed
    }
  } else if (K::kConv && warp >= kConvWarp0) {
    // --------------------------------------------------------- converters
    const int cw = warp - kConvWarp0;
    __shared__ float row_scale[kConvWarps][32];  // FP8: scale of stage row (pb*8 + k)
    // block count (-1: end of work, -2: not fetched yet) and (FP8) the row
    // scale of this lane's gathered row of an owned stage, probed one owned
    // stage ahead in the metadata ring (never waited for ahead of the stage
    // being converted: see the tile builders)
    bool ok = true;
    auto meta_of = [&](int64_t st, int& nb, float& sc, bool wait) {
      nb = -2;
      sc = 0.0f;
      const int ms = (int)(st % kMetaDepth);
      const uint32_t par = (uint32_t)(st / kMetaDepth) & 1;
      if (!wait) {
        if (!__all_sync(0xffffffffu, mbar_try_wait(&rings.meta_full[ms], par))) return;
      } else if (!warp_wait(&rings.meta_full[ms], par, p.err, abort_flag)) {
        ok = false;
        return;
      }
      nb = rings.meta[ms].nb;
      const int32_t r = rings.meta[ms].s2x[lane];
      __syncwarp();
      if (lane == 0) mbar_arrive(&rings.meta_empty[ms]);
      if (FORM == kFormFP8 && nb >= 0)
        sc = (lane < nb * BW && !((lane % BW) > 0 && r == 0))
                 ? __ldg(reinterpret_cast<const float*>(p.B1) + r) : 0.0f;
    };
    int nb_c, nb_n;
    float sc_c, sc_n;
    meta_of(cw, nb_c, sc_c, true);
    const int nchunk = ncols >> 3;  // 8-feature chunks per gathered row
    for (int64_t st = cw; ok && nb_c >= 0; st += kConvWarps) {
      meta_of(st + kConvWarps, nb_n, sc_n, false);
      const int s = (int)(st % S);
      const uint32_t n = (uint32_t)(st / S);
      const int nb = nb_c;
      if (!warp_wait(&loaded[s], n & 1, p.err, abort_flag)) break;  // implies the stage was empty
      if (FORM == kFormFP8) {
        row_scale[cw][lane] = sc_c;
        __syncwarp();
      }
      uint8_t* xs = xring + (size_t)s * K::kStageX;
      const uint8_t* es = ering + (size_t)s * K::kStageE;
      const int items = nb * BW * nchunk;
      // item it: 8 features (16 B of bf16) of gathered row rowi = pb * BW + k
      auto locate = [&](int it, uint32_t& xoff, uint32_t& eoff, int& rowi) {
        rowi = nchunk == NT * 16 ? it / (NT * 16) : it / nchunk;
        const int j = it - rowi * nchunk;
        const int pb = rowi / BW, k = rowi % BW;
        xoff = (uint32_t)(((pb * NT + (j >> 4)) * K::kSub + (k >> 3)) * kTileBytes) +
               x_offset_bf16(k & 7, j & 15);
        eoff = (uint32_t)(rowi * K::kRowStage + j * 8);
      };
      // SPLIT24: lo = b24 - hi is exact in bf16, so its bf16 bits are the
      // top half of the fp32 difference. Per element pair: the hi bits go
      // to the top of two fp32 words (byte permutes), the extension bytes
      // under them, one packed fp32x2 subtraction, one permute to pack.
      auto lo_words = [&](const uint4& h, const uint2& e, uint32_t (&o)[4]) {
        const uint32_t hw[4] = {h.x, h.y, h.z, h.w};
        const uint32_t ew[2] = {e.x, e.y};
#pragma unroll
        for (int z = 0; z < 4; ++z) {
          const uint32_t eword = ew[z >> 1];
          const uint32_t sel0 = 0x3200u | ((4u + 2u * (z & 1)) << 4);      // ext byte 2z
          const uint32_t sel1 = 0x3200u | ((4u + 2u * (z & 1) + 1u) << 4); // ext byte 2z+1
          const uint32_t h0 = __byte_perm(hw[z], 0u, 0x1044);
          const uint32_t h1 = hw[z] & 0xFFFF0000u;
          const uint32_t b0 = __byte_perm(h0, eword, sel0);
          const uint32_t b1 = __byte_perm(h1, eword, sel1);
          uint32_t l0, l1;
          asm("{\n\t.reg .b64 a, b, d;\n\t"
              "mov.b64 a, {%2, %3};\n\t"
              "mov.b64 b, {%4, %5};\n\t"
              "sub.rn.f32x2 d, a, b;\n\t"
              "mov.b64 {%0, %1}, d;\n\t}"
              : "=r"(l0), "=r"(l1)
              : "r"(b0), "r"(b1), "r"(h0), "r"(h1));
          o[z] = __byte_perm(l0, l1, 0x7632);
        }
      };
      auto fp8_words = [&](const uint2& e, float sc, uint32_t (&o)[4]) {
        const uint32_t ew[2] = {e.x, e.y};
#pragma unroll
        for (int z = 0; z < 4; ++z) {
          const uint16_t q2 = (uint16_t)(ew[z >> 1] >> ((z & 1) * 16));
          const __half2_raw hr = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)q2, __NV_E4M3);
          const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&hr));
          const __nv_bfloat162 b2 = __floats2bfloat162_rn(f.x * sc, f.y * sc);
          o[z] = *reinterpret_cast<const uint32_t*>(&b2);
        }
      };
      constexpr int U = 4;  // independent items per trip: all loads first, then math, then stores
      int it = lane;
      for (; it + 32 * (U - 1) < items; it += 32 * U) {
        uint32_t xo[U], eo[U];
        int ri[U];
        uint4 h[U];
        uint2 e[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          locate(it + 32 * u, xo[u], eo[u], ri[u]);
          e[u] = *reinterpret_cast<const uint2*>(es + eo[u]);
          if (FORM == kFormSplit24) h[u] = *reinterpret_cast<const uint4*>(xs + xo[u]);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
          uint32_t o[4];
          if (FORM == kFormSplit24) {
            lo_words(h[u], e[u], o);
            *reinterpret_cast<uint4*>(xs + xo[u] + 2048) = make_uint4(o[0], o[1], o[2], o[3]);
          } else {
            fp8_words(e[u], row_scale[cw][ri[u]], o);
            *reinterpret_cast<uint4*>(xs + xo[u]) = make_uint4(o[0], o[1], o[2], o[3]);
          }
        }
      }
      for (; it < items; it += 32) {
        uint32_t xo, eo;
        int ri;
        locate(it, xo, eo, ri);
        const uint2 e = *reinterpret_cast<const uint2*>(es + eo);
        uint32_t o[4];
        if (FORM == kFormSplit24) {
          lo_words(*reinterpret_cast<const uint4*>(xs + xo), e, o);
          *reinterpret_cast<uint4*>(xs + xo + 2048) = make_uint4(o[0], o[1], o[2], o[3]);
        } else {
          fp8_words(e, row_scale[cw][ri], o);
          *reinterpret_cast<uint4*>(xs + xo) = make_uint4(o[0], o[1], o[2], o[3]);
        }
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&full[s]);
      nb_c = nb_n;
      sc_c = sc_n;
      if (nb_c == -2) meta_of(st + kConvWarps, nb_c, sc_c, true);  // not ready when probed
    }
  } else if (warp >= kMmaWarp && warp < kMmaWarp + kMmaWarps) {
    // ------------------------------------------------------------- UMMA
    if (lane == 0) {
      const int m = warp - kMmaWarp;
      constexpr uint32_t idesc = umma_idesc(1, 128, 2 * WH, 1, 0);
      const uint64_t adesc0 = umma_desc(smem_u32(xring), 1024, 2048, 2);
      const uint64_t bdesc0 = umma_desc(smem_u32(yring), 128, 256, 0);
      const uint32_t adesc_lo = (uint32_t)adesc0, adesc_hi = (uint32_t)(adesc0 >> 32);
      const uint32_t bdesc_lo = (uint32_t)bdesc0, bdesc_hi = (uint32_t)(bdesc0 >> 32);
      uint32_t q = 0;
      bool ok = true;
      for (uint32_t rq = 0; ok; ++rq) {
        const int rs = (int)(rq % kRecDepth);
        if (!mbar_wait(&rings.rec_full[rs], (rq / kRecDepth) & 1, p.err)) { ok = false; break; }
        const WinRec rec = rings.rec[rs];
        mbar_arrive(&rings.rec_empty[rs]);
        if (rec.flags & kRecEnd) break;
        if (rec.flags & kRecEmpty) continue;
        if (rec.flags & kRecPad) {  // a stage without blocks: its owner passes it on
          if ((int)(rec.stage_base & 1) == m) {
            const int s = (int)(rec.stage_base % S);
            if (!mbar_wait(&full[s], (uint32_t)(rec.stage_base / S) & 1, p.err)) { ok = false; break; }
            mbar_arrive(&empty[s]);
          }
          continue;
        }
        const int a = (int)(q % K::kNacc);
        if (!mbar_wait(&acc_empty[a], ((q / K::kNacc) & 1) ^ 1, p.err)) { ok = false; break; }
        tc_fence_after();
        const uint32_t dtm = tmem_base + (uint32_t)((m * K::kNacc + a) * K::kAccCols);
        uint32_t acc = 0;
        // this issuer's stages of the window, in order (stage g belongs to
        // issuer g % 2; chunks start on even stages, so the chunk-relative
        // index gives the same issuer). Indices relative to the chunk fit 32 bits
        // (T < 2^31); the CTA's stage counter is kept modulo 2^32, which S divides.
        const int32_t rb0 = (int32_t)(rec.wb0 - rec.cb0), rb1 = (int32_t)(rec.wb1 - rec.cb0);
        const int32_t cbn = (int32_t)(rec.cb1 - rec.cb0);
        int32_t rel = rb0 / P;
        rel += (int32_t)((rel & 1) != m);
        uint32_t g = (uint32_t)rec.stage_base + (uint32_t)rel;
        for (int32_t sbr = rel * P; sbr < rb1; sbr += kMmaWarps * P, g += kMmaWarps) {
          const int s = (int)(g % S);
          const int32_t lo = sbr > rb0 ? sbr : rb0;
          const int32_t hi = (sbr + P) < rb1 ? (sbr + P) : rb1;
          if (lo == sbr) {  // first visit of this stage (windows are walked in order)
            if (!mbar_wait(&full[s], (g / S) & 1, p.err)) { ok = false; break; }
            fence_proxy_async_smem();  // cp.async (generic proxy) data -> UMMA reads
            tc_fence_after();
          }
          uint32_t blo = bdesc_lo + (uint32_t)((s * K::kStageY + (lo - sbr) * K::kYB) >> 4);
          uint32_t alo = adesc_lo + (uint32_t)((s * K::kStageX + (lo - sbr) * NT * K::kSub * kTileBytes) >> 4);
#pragma unroll
          for (int j = 0; j < P; ++j) {
            if (lo + j < hi) {
#pragma unroll
              for (int h = 0; h < K::kSub; ++h)
#pragma unroll
                for (int t = 0; t < NT; ++t)
                  mma_f16(dtm + t * 2 * WH,
                           desc_at(alo + (uint32_t)(((t * K::kSub + h) * kTileBytes) >> 4), adesc_hi),
                           desc_at(blo + (uint32_t)((h * K::kYB8) >> 4), bdesc_hi), idesc,
                           h == 0 ? acc : 1u);
              acc = 1;
              alo += (uint32_t)((NT * K::kSub * kTileBytes) >> 4);
              blo += (uint32_t)(K::kYB >> 4);
            }
          }
          if (hi == sbr + P || hi == cbn) tc_commit(&empty[s]);  // stage fully consumed
        }
        if (!ok) break;
        tc_commit(&acc_full[a]);
        ++q;
      }
      if (!ok) *abort_flag = 1;
      // every MMA this thread issued has finished before the CTA frees TMEM
      // (also when a wait gave up with MMAs in flight)
      tc_commit(&drain[m]);
      mbar_wait(&drain[m], 0, p.err);
    }
    __syncwarp();
  } else if (warp < kEpiWarps) {
    // --------------------------------------------------------- epilogue
    const int ew = warp;
    uint32_t q = 0;
    uint32_t su = 0;  // C tiles this warp has staged (selects the staging buffer)
    for (uint32_t rq = 0;; ++rq) {
      const int rs = (int)(rq % kRecDepth);
      if (!warp_wait(&rings.rec_full[rs], (rq / kRecDepth) & 1, p.err, abort_flag)) break;
      const WinRec rec = rings.rec[rs];
      __syncwarp();
      if (lane == 0) mbar_arrive(&rings.rec_empty[rs]);
      if (rec.flags & kRecEnd) break;
      if (rec.flags & kRecPad) continue;
      if (rec.flags & kRecEmpty) {
        zero_window_rows(p, rec.w, col0, ncols, ew * 32 + lane, 32 * kEpiWarps);
        continue;
      }
      const int a = (int)(q % K::kNacc);
      if (!warp_wait(&acc_full[a], (q / K::kNacc) & 1, p.err, abort_flag)) break;
      tc_fence_after();
      const int64_t row0 = (int64_t)rec.w * WH;
      float* out;
      bool guard_rows = true;
      if (p.mode == 1 && (rec.flags & (kRecHead | kRecTail))) {
        const int slot = (rec.flags & kRecHead) ? 2 * rec.chunk : 2 * rec.chunk + 1;
        out = p.part + (size_t)slot * WH * p.N;
        guard_rows = false;
      } else {
        out = p.C + row0 * p.N;
      }
      const int64_t st0 = (rec.wb0 - rec.cb0) / P, st1 = (rec.wb1 - 1 - rec.cb0) / P;
      const bool both = st1 > st0;
      const int m0 = (int)(st0 % kMmaWarps);
      const uint32_t lane_addr = tmem_base + ((uint32_t)(ew * 32) << 16);
#pragma unroll 1
      for (int t = 0; t < NT; ++t) {
        const int f = col0 + t * 128 + ew * 32 + lane;
#pragma unroll 1
        for (int h = 0; h < WH / 16; ++h) {  // 16 window rows at a time
          float x[16];
#pragma unroll
          for (int r = 0; r < 16; ++r) x[r] = 0.0f;
          // fixed order: issuer 0's partial, then issuer 1's
#pragma unroll 1
          for (int mi = 0; mi < kMmaWarps; ++mi) {
            if (!both && mi != m0) continue;
            uint32_t v[16], u[16];
            const uint32_t col = (uint32_t)((mi * K::kNacc + a) * K::kAccCols + t * 2 * WH);
            tmem_ld16(lane_addr + col + h * 16, v);       // A_hi columns
            tmem_ld16(lane_addr + col + WH + h * 16, u);  // A_lo columns
            tmem_ld_wait();
#pragma unroll
            for (int r = 0; r < 16; ++r) x[r] += __uint_as_float(v[r]) + __uint_as_float(u[r]);
          }
          if (t == NT - 1 && h == WH / 16 - 1) {
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[a]);
          }
          if (!guard_rows) {  // partial tile of a cut window: raw sums to the workspace
            if (f < p.N) {
              float* o = out + (size_t)h * 16 * p.N;
#pragma unroll
              for (int r = 0; r < 16; ++r) o[r * p.N + f] = x[r];
            }
          } else if (col0 + t * 128 + ew * 32 < p.N) {
            // finished 16-row tile of this warp's 32 columns: shared memory, then
            // one TMA store (rows past M and columns past N are clipped)
            float* sb = reinterpret_cast<float*>(stg + (ew * 2 + (su & 1)) * K::kStgW);
            __syncwarp();  // lane 0 has waited for this buffer's previous store
#pragma unroll
            for (int r = 0; r < 16; ++r) sb[r * 32 + lane] = epilogue(p, x[r], f < p.N ? f : 0);
            fence_proxy_async_smem();
            __syncwarp();
            if (lane == 0) {
              tma_store_2d(&p.cmap, sb, col0 + t * 128 + ew * 32, (int32_t)(row0 + h * 16));
              bulk_commit();
              bulk_wait_read<1>();
            }
            ++su;
          }
        }
      }
      ++q;
    }
    if (lane == 0) bulk_wait_all();
  }

  tc_fence_before();
  __syncthreads();
  if (threadIdx.x == 0 && p.stamps) {
    uint32_t smid;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
    record_cta_time(p, 0, t_entry);
    record_cta_time(p, 1, global_timer_ns());
    record_cta_time(p, 2, smid);
  }
  if (warp == kMmaWarp) {
    tc_fence_after();
    tmem_dealloc(tmem_base, K::kTmemCols);
  }
}

template <int FORM, int NT, int P, int S, bool FOUR, int WH, int BW>
dtc_status launch_split(const Params& p, int slices, cudaStream_t st) {
  using K = SCfg<FORM, NT, P, S, WH, BW>;
  constexpr int smem = K::kSmem;
  static_assert(smem <= 227 * 1024, "shared memory budget");
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    DTC_CUDA(cudaFuncSetAttribute(k_spmm_split<FORM, NT, P, S, FOUR, WH, BW>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr_set[dev & 63] = true;
  }
  dim3 grid((unsigned)launch_ctas(p, slices), (unsigned)slices);
  k_spmm_split<FORM, NT, P, S, FOUR, WH, BW><<<grid, K::kThreads, smem, st>>>(p);
  DTC_CUDA(cudaGetLastError());
  if (p.mode == 1 && p.G > 1) {
    k_reduce_partials<<<p.G - 1, 256, 0, st>>>(p);
    DTC_CUDA(cudaGetLastError());
  }
  return DTC_OK;
}

// N-tiles per CTA: all of N up to 4 (window height 16) or 2 (height 32, whose
// accumulators are twice as wide) unless capped by `ntile`.
template <int FORM, bool FOUR>
dtc_status dispatch_n(const Params& p, int nt, int W, int slices, cudaStream_t st) {
  if (W == 16) {  // 16 gathered rows per block: half the blocks per stage
    if (nt == 1) return launch_split<FORM, 1, 2, 8, FOUR, 16, 16>(p, slices, st);
    return launch_split<FORM, 2, 1, 8, FOUR, 16, 16>(p, slices, st);
  }
  if (p.H == 32) {
    // forms with a staging ring for the second plane hold 3 blocks per stage so
    // the 32-row A tiles fit in shared memory; the others keep 4
    constexpr int P32 = (FORM == kFormBF16 || FORM == kFormBF16X2) ? 4 : 3;
    if (nt == 1) return launch_split<FORM, 1, P32, 8, FOUR, 32, 8>(p, slices, st);
    return launch_split<FORM, 2, 2, 8, FOUR, 32, 8>(p, slices, st);
  }
  if (nt == 1) return launch_split<FORM, 1, 4, 8, FOUR, 16, 8>(p, slices, st);
  if (nt == 2) return launch_split<FORM, 2, 2, 8, FOUR, 16, 8>(p, slices, st);
  return launch_split<FORM, 4, 1, 8, FOUR, 16, 8>(p, slices, st);
}

}  // namespace

dtc_status spmm_split_impl(const int32_t* rwo, const uint8_t* tile, const int32_t* toff,
                           const int32_t* s2x, const float* vals, int32_t M, int32_t nwin,
                           int64_t T, int bformat, const void* p0, const void* p1, int32_t N,
                           int precision, float* C, int mode, int grid, float* part,
                           cudaStream_t st, int ntile, Epilogue epi, int H, void* queue,
                           int W) {
  DTC_REQUIRE(M >= 0 && N >= 1 && T >= 0, "bad sizes");
  DTC_REQUIRE(T < ((int64_t)1 << 31), "more than 2^31 - 1 TC blocks");
  DTC_REQUIRE(bformat == DTC_B_SPLIT24 || bformat == DTC_B_BF16 || bformat == DTC_B_FP8 ||
                  bformat == DTC_B_BF16X2,
              "split kernels take SPLIT24, BF16, FP8 or BF16X2 B");
  DTC_REQUIRE(precision == DTC_PREC_SPLIT3 || precision == DTC_PREC_SPLIT4,
              "split kernels take precision SPLIT3 or SPLIT4");
  DTC_REQUIRE(N % 16 == 0, "split forms need N % 16 == 0 (16-byte row segments of every plane)");
  DTC_REQUIRE(bformat == DTC_B_BF16 || p1 != nullptr, "second B plane missing");
  DTC_REQUIRE(((uintptr_t)p0 & 15) == 0 && ((uintptr_t)p1 & 15) == 0, "planes must be 16-byte aligned");
  DTC_REQUIRE(((uintptr_t)s2x & 15) == 0, "SparseAToX must be 16-byte aligned");
  DTC_REQUIRE(H == 16 || H == 32, "window height must be 16 or 32");
  DTC_REQUIRE(W == 8 || (W == 16 && H == 16),
              "block width must be 8, or 16 at window height 16 (tile ids are bytes)");
  DTC_REQUIRE(nwin == (M + H - 1) / H, "num_windows must be ceil(num_nodes / window height)");
  DTC_REQUIRE(mode == 0 || part != nullptr, "balance mode needs the partials workspace");
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
  p.B = reinterpret_cast<const float*>(p0); p.B1 = p1; p.bformat = bformat;
  p.C = C; p.part = part; p.err = device_error_word();
  p.bias = epi.bias; p.relu = epi.relu;
  p.M = M; p.nwin = nwin; p.N = N; p.T = T; p.mode = mode; p.H = H;
  DTC_REQUIRE(((uintptr_t)C & 15) == 0, "C must be 16-byte aligned");
  dtc_status es = encode_c_map(&p.cmap, C, M, N, 16);
  if (es != DTC_OK) return es;
  int G = grid > 0 ? grid : default_chunks();
  if ((int64_t)G > T) G = (int)T;
  p.G = G;
  int nt = N <= 128 ? 1 : N <= 256 ? 2 : 4;
  if (ntile == 1 || ntile == 2) nt = nt < ntile ? nt : ntile;
  if ((H == 32 || W == 16) && nt > 2) nt = 2;
  const int slices = (N + nt * 128 - 1) / (nt * 128);
  es = setup_queue(p, queue, slices, st);
  if (es != DTC_OK) return es;
  const bool four = precision == DTC_PREC_SPLIT4;
  switch (bformat) {
    case DTC_B_SPLIT24:
      return four ? dispatch_n<kFormSplit24, true>(p, nt, W, slices, st)
                  : dispatch_n<kFormSplit24, false>(p, nt, W, slices, st);
    case DTC_B_BF16:
      return four ? dispatch_n<kFormBF16, true>(p, nt, W, slices, st)
                  : dispatch_n<kFormBF16, false>(p, nt, W, slices, st);
    case DTC_B_BF16X2:
      return four ? dispatch_n<kFormBF16X2, true>(p, nt, W, slices, st)
                  : dispatch_n<kFormBF16X2, false>(p, nt, W, slices, st);
    default:
      return four ? dispatch_n<kFormFP8, true>(p, nt, W, slices, st)
                  : dispatch_n<kFormFP8, false>(p, nt, W, slices, st);
  }
}

}  // namespace dtc
