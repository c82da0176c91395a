// TC-block SpMM on sm_100a: cp.async gathers of dense rows into swizzled
// shared memory, tcgen05.mma into TMEM, warp-specialised persistent CTAs fed
// by a producer warp, deterministic strict balance.
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
// Work split and determinism: see spmm_sched.cuh (chunks of the TC-block
// range, a chunk queue, partial tiles indexed by chunk).
//
// Pipeline. A ring of S stages, each holding P consecutive TC blocks of a
// chunk (barrier traffic is per stage, not per block).
//   warps 0-3   epilogue: walks the window records; tcgen05.ld 32x32b; each
//               warp stages its 32 columns x window rows of C in shared memory
//               and issues one TMA tensor store (plain per-lane stores stalled
//               these warps and, through the accumulator hand-off, the whole
//               pipeline); empty windows get zero rows
//   warps 4-5   UMMA issuers (one thread each; warp 4 also owns TMEM): issuer
//               m takes the chunk-relative stages s % 2 == m into its own set
//               of accumulators, so two MMA streams are in flight (a single
//               issuing thread cannot saturate the tensor pipe with these
//               small M128 x N16 x K8 instructions); the epilogue adds the two
//               partial accumulators in a fixed order
//   warps 6-9   loaders: cp.async 16-byte gathers of B rows (SparseAToX from
//               the stage's metadata slot), zero-fill for padded slots; stage
//               s is owned by loader s % 4
//   warps 10-13 tile builders: zero + scatter TC-block values into A_b^T;
//               stage s is owned by tile builder s % 4; tile ids and values
//               are loaded two owned stages ahead from the offsets in the
//               metadata ring
//   warp 14     producer (spmm_sched.cuh): chunk claims, stage metadata,
//               window records
// Every data-ring and metadata-ring wait is by a warp on its own residue
// class of stages, in order (a parity wait more than one phase ahead would
// pass spuriously). Every wait is bounded (2 s) and records kErrWaitTimeout
// instead of hanging.
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
constexpr int kProdWarp = kTileWarp0 + kTileWarps;
constexpr int kThreads = 32 * (kProdWarp + 1);  // 480
constexpr int kXTileBytes = 4096;   // 8 rows x 128 fp32 features

// Byte offset, inside one 8-row x 128-feature fp32 tile, of 16-byte chunk
// `cc` (features 4cc..4cc+3) of row k, in the UMMA layout-type-1 atom order:
// atom = 32 features x 4 rows (512 B), 32-byte granule index XOR (row & 3).
__device__ __forceinline__ uint32_t x_offset_tf32(uint32_t k, uint32_t cc) {
  const uint32_t a = cc >> 3, j = cc & 7;
  const uint32_t g = (j >> 1) ^ (k & 3);
  return a * 1024 + (k >> 2) * 512 + (k & 3) * 128 + ((g << 1) | (j & 1)) * 16;
}

// WH = row-window height (the UMMA N dimension): 16 or 32. BW = TC-block
// width (compaction width, 8 or 16): a block of width 16 is two 8-slot halves,
// each its own K = 8 MMA into the same accumulator.
template <int NT, int P, int S, int WH, int BW>
struct Cfg {
  static_assert(S % kLoadWarps == 0 && S % kTileWarps == 0, "stage ownership");
  static_assert(kLoadWarps <= kEndStages && kTileWarps <= kEndStages, "end markers");
  static_assert(BW == 8 || BW == 16, "block width");
  static_assert((S & (S - 1)) == 0 && S % 2 == 0, "stage counters are kept modulo 2^32");
  static_assert(P * BW <= 32, "one SparseAToX entry per lane");
  static_assert(WH * BW <= 256, "tile ids are bytes");
  static_assert(P + 1 <= 8, "stage offsets fit the metadata slot");
  static_assert(WH == 16 || WH == 32, "window height");
  static constexpr int kSub = BW / 8;                   // 8-slot halves per block
  static constexpr int kNacc = (NT * WH > 64) ? 2 : 4;  // TMEM accumulator buffers in flight
  static constexpr int kYB8 = WH * 8 * 4;               // WH x 8 fp32, K-major core matrices
  static constexpr int kYB = kSub * kYB8;               // one block's A^T tile
  static constexpr int kStageX = P * NT * kSub * kXTileBytes;
  static constexpr int kStageY = P * kYB;
  static constexpr int kX = S * kStageX;
  static constexpr int kY = S * kStageY;
  static constexpr int kStgW = WH * 32 * 4;               // one epilogue warp's C tile
  static constexpr int kStg = kEpiWarps * 2 * kStgW;       // double-buffered per warp
  static constexpr int kBars = (2 * S + 2 * kNacc + kMmaWarps) * 8;
  static constexpr int kSmem = kX + kY + kStg + kSchedBytes + kBars + 16 + 1024;
  static_assert(kSmem <= 232448, "dynamic shared memory per CTA");
  static constexpr int kCols = kMmaWarps * kNacc * NT * WH;  // TMEM columns used
  static_assert(kCols <= 512, "TMEM budget");
  static constexpr uint32_t kTmemCols = kCols <= 32 ? 32 : kCols <= 64 ? 64 : kCols <= 128 ? 128
                                        : kCols <= 256 ? 256 : 512;
};

template <int NT, int P, int S, int WH, int BW>
__global__ void __launch_bounds__(kThreads, 1) k_spmm_tf32(const __grid_constant__ Params p) {
  using K = Cfg<NT, P, S, WH, BW>;
  const uint64_t t_entry = global_timer_ns();
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  uint8_t* xring = smem;
  uint8_t* yring = smem + K::kX;
  uint8_t* stg = yring + K::kY;          // [4 warps][2][WH x 32] fp32 C staging
  const SchedRings rings = carve_rings(stg + K::kStg);
  uint64_t* bars = (uint64_t*)(stg + K::kStg + kSchedBytes);
  uint64_t* full = bars;                 // [S] 32 cp.async arrivals + 1 tile arrival
  uint64_t* empty = bars + S;            // [S] the owning issuer's UMMA commit
  uint64_t* acc_full = bars + 2 * S;     // [kNacc] UMMA commit
  uint64_t* acc_empty = acc_full + K::kNacc;  // [kNacc] 4 epilogue warps
  uint64_t* drain = acc_empty + K::kNacc;     // [kMmaWarps] an issuer's last commit
  uint32_t* tmem_slot = (uint32_t*)(drain + kMmaWarps);
  volatile uint32_t* abort_flag = tmem_slot + 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int col0 = blockIdx.y * NT * 128;      // this CTA's feature slice
  const int ncols = (p.N - col0) < NT * 128 ? (p.N - col0) : NT * 128;
  const int nck = ncols >> 2;                  // 16-byte chunks per gathered row

  if (threadIdx.x == 0) {
    for (int i = 0; i < S; ++i) {
      mbar_init(&full[i], 32 + 1);
      mbar_init(&empty[i], 1);  // the owning issuer's MMA commit
    }
    for (int i = 0; i < K::kNacc; ++i) {
      mbar_init(&acc_full[i], kMmaWarps);
      mbar_init(&acc_empty[i], kEpiWarps);
    }
    for (int i = 0; i < kMmaWarps; ++i) mbar_init(&drain[i], 1);
    // metadata: loader + tile builder; records: every epilogue warp and issuer
    init_rings(rings, 2, kEpiWarps + kMmaWarps);
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

  if (warp == kProdWarp) {
    produce<P, BW, kMmaWarps>(p, rings, lane, abort_flag);
  } else if (warp >= kLoadWarp0 && warp < kLoadWarp0 + kLoadWarps) {
    // ------------------------------------------------------------ loaders
    const int lw = warp - kLoadWarp0;
    __shared__ int32_t rows_sm[kLoadWarps][32];  // SparseAToX of the stage being loaded
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
      if (nck == NT * 32) {
        // full 128-feature tiles: one gathered row per warp instruction
        for (int pb = 0; pb < nb; ++pb) {
#pragma unroll
          for (int k = 0; k < BW; ++k) {
            const int32_t r = __shfl_sync(0xffffffffu, rows, pb * BW + k);
            const bool pad = (k > 0 && r == 0);  // unused slot (columns ascend in a block)
            const float* src = p.B + (int64_t)(pad ? 0 : r) * p.N + col0;
#pragma unroll
            for (int t = 0; t < NT; ++t)
              cp_async16(xs + ((pb * NT + t) * K::kSub + (k >> 3)) * kXTileBytes +
                             x_offset_tf32(k & 7, lane),
                         src + (t * 32 + lane) * 4, pad ? 0u : 16u);
          }
        }
      } else if (nck == 16 || nck == 8) {
        // 64- or 32-feature rows: 32 / nck gathered rows per warp instruction
        const int lg = nck == 16 ? 4 : 3;
        const int sub = lane >> lg, cc = lane & (nck - 1);
        for (int pb = 0; pb < nb; ++pb) {
          for (int k0 = 0; k0 < BW; k0 += 32 >> lg) {
            const int k = k0 + sub;
            const int32_t r = __shfl_sync(0xffffffffu, rows, pb * BW + k);
            const bool pad = (k > 0 && r == 0);
            const float* src = p.B + (int64_t)(pad ? 0 : r) * p.N + col0;
            cp_async16(xs + (pb * NT * K::kSub + (k >> 3)) * kXTileBytes + x_offset_tf32(k & 7, cc),
                       src + cc * 4, pad ? 0u : 16u);
          }
        }
      } else {
        // partial slice: lanes flattened over (gathered row, 16-byte chunk)
        rows_sm[lw][lane] = rows;
        __syncwarp();
        for (int idx = lane; idx < nb * BW * nck; idx += 32) {
          const int rowi = idx / nck, cc = idx - rowi * nck;
          const int k = rowi % BW, pb = rowi / BW;
          const int32_t r = rows_sm[lw][rowi];
          const bool pad = (k > 0 && r == 0);
          const float* src = p.B + (int64_t)(pad ? 0 : r) * p.N + col0;
          cp_async16(xs + ((pb * NT + (cc >> 5)) * K::kSub + (k >> 3)) * kXTileBytes +
                         x_offset_tf32(k & 7, cc & 31),
                     src + cc * 4, pad ? 0u : 16u);
        }
        __syncwarp();
      }
      cp_async_arrive_noinc(&full[s]);
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
        const uint32_t pos = i == 0 ? cur.t0 : i == 1 ? cur.t1 : __ldg(p.tile + e);
        const float v = i == 0 ? cur.v0 : i == 1 ? cur.v1 : (p.vals ? __ldg(p.vals + e) : 1.0f);
        if (pos < WH * BW) {
          if (v != 0.0f) {
            uint32_t t32;
            asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(t32) : "f"(v));
            const uint32_t r = pos / BW, sl = pos % BW;
            *reinterpret_cast<uint32_t*>(ys + pb * K::kYB + (sl >> 3) * K::kYB8 +
                                         y_offset(r * 8 + (sl & 7))) = t32;
          }
        } else {
          atomicOr(p.err, kErrBadIndex);
        }
      }
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0) mbar_arrive(&full[s]);
      cur = n1;
      n1 = n2;
      if (cur.nb == -2) fetch(st + kTileWarps, cur, true);  // not ready when probed
    }
  } else if (warp >= kMmaWarp && warp < kMmaWarp + kMmaWarps) {
    // ------------------------------------------------------------- UMMA
    if (lane == 0) {
      const int m = warp - kMmaWarp;  // this issuer's stages: chunk-relative index % 2 == m
      constexpr uint32_t idesc = umma_idesc(2, 128, WH, 1, 0);
      // Descriptors advance by adding (byte offset >> 4) to the start-address
      // field (shared addresses < 256 KB fit its 14 bits, no carry out).
      const uint64_t adesc0 = umma_desc(smem_u32(xring), 1024, 512, 1);
      const uint64_t bdesc0 = umma_desc(smem_u32(yring), 128, 256, 0);
      const uint32_t adesc_lo = (uint32_t)adesc0, adesc_hi = (uint32_t)(adesc0 >> 32);
      const uint32_t bdesc_lo = (uint32_t)bdesc0, bdesc_hi = (uint32_t)(bdesc0 >> 32);
      uint32_t q = 0;        // nonempty windows met
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
        const uint32_t dtm = tmem_base + (uint32_t)((m * K::kNacc + a) * NT * WH);
        uint32_t acc = 0;
        // this issuer's stages of the window, in order (stage g belongs to
        // issuer g % 2; chunks start on even stages, so the chunk-relative
        // index has the same parity). Indices relative to the chunk fit 32 bits
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
          uint32_t alo = adesc_lo + (uint32_t)((s * K::kStageX + (lo - sbr) * NT * K::kSub * kXTileBytes) >> 4);
#pragma unroll
          for (int j = 0; j < P; ++j) {
            if (lo + j < hi) {
#pragma unroll
              for (int h = 0; h < K::kSub; ++h)
#pragma unroll
                for (int t = 0; t < NT; ++t)
                  mma_tf32(dtm + t * WH,
                           desc_at(alo + (uint32_t)(((t * K::kSub + h) * kXTileBytes) >> 4), adesc_hi),
                           desc_at(blo + (uint32_t)((h * K::kYB8) >> 4), bdesc_hi), idesc,
                           h == 0 ? acc : 1u);
              acc = 1;
              alo += (uint32_t)((NT * K::kSub * kXTileBytes) >> 4);
              blo += (uint32_t)(K::kYB >> 4);
            }
          }
          if (hi == sbr + P || hi == cbn) tc_commit(&empty[s]);  // stage fully consumed
        }
        if (!ok) break;
        tc_commit(&acc_full[a]);  // also when this issuer had no block in the window
        ++q;
      }
      if (!ok) *abort_flag = 1;
      // every MMA this thread issued has finished before the CTA frees TMEM
      // (also when a wait gave up with MMAs in flight)
      tc_commit(&drain[m]);
      mbar_wait(&drain[m], 0, p.err);
    }
    __syncwarp();
  } else {
    // --------------------------------------------------------- epilogue
    const int ew = warp;  // TMEM lanes 32*ew .. 32*ew+31
    uint32_t q = 0;
    uint32_t su = 0;      // C tiles this warp has staged (selects the staging buffer)
    for (uint32_t rq = 0;; ++rq) {
      const int rs = (int)(rq % kRecDepth);
      if (!warp_wait(&rings.rec_full[rs], (rq / kRecDepth) & 1, p.err, abort_flag)) break;
      const WinRec rec = rings.rec[rs];
      __syncwarp();
      if (lane == 0) mbar_arrive(&rings.rec_empty[rs]);
      if (rec.flags & kRecEnd) break;
      if (rec.flags & kRecPad) continue;
      if (rec.flags & kRecEmpty) {  // empty window: C rows are zero
        zero_window_rows(p, rec.w, col0, ncols, ew * 32 + lane, 32 * kEpiWarps);
        continue;
      }
      const int a = (int)(q % K::kNacc);
      if (!warp_wait(&acc_full[a], (q / K::kNacc) & 1, p.err, abort_flag)) break;
      tc_fence_after();
      const int64_t row0 = (int64_t)rec.w * WH;
      float* out;
      bool guard_rows = true;
      if (p.mode == 1 && (rec.flags & (kRecHead | kRecTail))) {  // window cut by a chunk boundary
        const int slot = (rec.flags & kRecHead) ? 2 * rec.chunk : 2 * rec.chunk + 1;
        out = p.part + (size_t)slot * WH * p.N;
        guard_rows = false;
      } else {
        out = p.C + row0 * p.N;
      }
      // issuers that hold part of this window: chunk-relative stages mod kMmaWarps
      const int64_t st0 = (rec.wb0 - rec.cb0) / P, st1 = (rec.wb1 - 1 - rec.cb0) / P;
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

template <int NT, int P, int S, int WH, int BW>
dtc_status launch_tf32(const Params& p, int slices, cudaStream_t st) {
  constexpr int smem = Cfg<NT, P, S, WH, BW>::kSmem;
  static_assert(smem <= 227 * 1024, "shared memory budget");
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    DTC_CUDA(cudaFuncSetAttribute(k_spmm_tf32<NT, P, S, WH, BW>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    attr_set[dev & 63] = true;
  }
  dim3 grid((unsigned)launch_ctas(p, slices), (unsigned)slices);
  k_spmm_tf32<NT, P, S, WH, BW><<<grid, kThreads, smem, st>>>(p);
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
                          float* part, cudaStream_t st, int ntile, Epilogue epi, int H,
                          void* queue, int W) {
  DTC_REQUIRE(M >= 0 && N >= 1 && T >= 0, "bad sizes");
  DTC_REQUIRE(T < ((int64_t)1 << 31), "more than 2^31 - 1 TC blocks");
  DTC_REQUIRE(N % 4 == 0, "tcgen05 path needs N % 4 == 0 (16-byte row segments)");
  DTC_REQUIRE(((uintptr_t)B & 15) == 0, "B must be 16-byte aligned");
  DTC_REQUIRE(((uintptr_t)s2x & 15) == 0, "SparseAToX must be 16-byte aligned");
  DTC_REQUIRE(H == 16 || H == 32, "window height must be 16 or 32");
  DTC_REQUIRE(W == 8 || (W == 16 && H == 16),
              "block width must be 8, or 16 at window height 16 (tile ids are bytes)");
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
  int G = grid > 0 ? grid : default_chunks();
  if ((int64_t)G > T) G = (int)T;
  p.G = G;
  // N-tiles (128 features each) per CTA: all of N up to 4 tiles unless capped
  // by `ntile`; wider slices of N go to more CTAs (grid.y).
  int nt = N <= 128 ? 1 : N <= 256 ? 2 : 4;
  if (ntile == 1 || ntile == 2) nt = nt < ntile ? nt : ntile;
  const int slices = (N + nt * 128 - 1) / (nt * 128);
  es = setup_queue(p, queue, slices, st);
  if (es != DTC_OK) return es;
  if (W == 16) {  // 16 gathered rows per block: half the blocks per stage
    if (nt == 1) return launch_tf32<1, 2, 8, 16, 16>(p, slices, st);
    if (nt == 2) return launch_tf32<2, 1, 8, 16, 16>(p, slices, st);
    return launch_tf32<4, 1, 4, 16, 16>(p, slices, st);
  }
  if (H == 32) {
    if (nt == 1) return launch_tf32<1, 4, 8, 32, 8>(p, slices, st);
    if (nt == 2) return launch_tf32<2, 2, 8, 32, 8>(p, slices, st);
    return launch_tf32<4, 1, 8, 32, 8>(p, slices, st);
  }
  if (nt == 1) return launch_tf32<1, 4, 8, 16, 8>(p, slices, st);
  if (nt == 2) return launch_tf32<2, 2, 8, 16, 8>(p, slices, st);
  return launch_tf32<4, 1, 8, 16, 8>(p, slices, st);
}

size_t spmm_partials_bytes(int64_t T, int32_t N, int grid, int H) {
  int G = grid > 0 ? grid : default_chunks();
  if ((int64_t)G > T) G = (int)(T > 0 ? T : 1);
  return (size_t)2 * G * H * (size_t)N * sizeof(float);
}

size_t spmm_queue_bytes(int64_t T, int grid) {
  int G = grid > 0 ? grid : default_chunks();
  if ((int64_t)G > T) G = (int)(T > 0 ? T : 1);
  return kQueueHeader + chunk_table_bytes(G);
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
