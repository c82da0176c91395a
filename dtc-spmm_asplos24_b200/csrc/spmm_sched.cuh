// Scheduling pieces shared by the TC-block SpMM kernels (tf32 and split
// precision): kernel parameters, the chunk work queue, the producer warp that
// feeds the stage-metadata and window-record rings, the A-tile layout,
// cp.async helpers and the deterministic partial reduction.
//
// Work split. The TC blocks [0, T) are cut into G chunks, chunk k covering
// blocks [k*T/G, (k+1)*T/G) (strict balance, mode 1) or that range snapped to
// row-window starts (window mode 0, windows never split). G is the split
// threshold knob: ceil(T / G) blocks per chunk. Two launch shapes share one
// kernel:
//   persistent  one CTA per SM (per N-slice); CTAs pull chunk ids from a
//               device counter (a global work queue), so a CTA that drew a
//               heavy chunk simply claims fewer; needs the small per-call
//               workspace that holds the counter and the per-chunk table
//   one-shot    one CTA per chunk (no workspace), the hardware block scheduler
//               hands out chunks as CTAs retire
// Results depend only on the chunking: windows cut by chunk boundaries write
// fp32 partial tiles to slots indexed by chunk id and k_reduce_partials sums
// them in chunk order, and inside a chunk the stage-to-issuer assignment is
// chunk-relative, so which CTA ran which chunk never changes a bit.
//
// Stage ownership. Stage g of a CTA (its g-th stage overall) sits in ring slot
// g % S and belongs to UMMA issuer g % I, I the kernel's issuer count (S is a
// multiple of I, so each issuer only ever meets its own slots, and only the
// owner waits on and releases a slot). Every chunk starts on a multiple of I:
// before a chunk that would start elsewhere, the producer emits pad stages (no
// blocks) with one kRecPad record each, which their owners wait on and
// release. A stage's issuer inside a chunk is therefore its chunk-relative
// index % I, whatever chunks the CTA ran before.
//
// Producer warp. One warp walks the CTA's chunks ahead of everyone else:
//   stage metadata  per stage of P consecutive blocks: first block, block
//                   count, TCblockoffset[sb .. sb+nb] and SparseAToX of the
//                   stage, copied by cp.async into a kMetaDepth-deep ring, so
//                   loaders and tile builders read their per-stage metadata
//                   from shared memory instead of waiting on global loads
//   window records  one per row window met in the chunk (empty windows
//                   included, which only the chunk owning their start block
//                   reports): window id, its blocks inside the chunk and
//                   whether a chunk boundary cuts it; the UMMA issuers and the
//                   epilogue walk windows from this ring
// The producer finds window boundaries from RowWindowOffset held 32 entries at
// a time in its lanes (one coalesced load per 31 windows, the next batch
// loaded ahead).
#pragma once
#include "common.cuh"

namespace dtc {
namespace {

constexpr int kMetaDepth = 16;    // stage-metadata ring (stages)
constexpr int kRecDepth = 32;     // window-record ring
constexpr int kEndStages = 8;     // end markers: one per residue class of the widest consumer role
constexpr int kEmitBatch = 4;     // stages the producer emits per pass
constexpr int kWavesPerSm = 16;   // default chunks per SM
constexpr size_t kQueueHeader = 256;  // workspace bytes holding the queue counters
inline int default_chunks() { return kWavesPerSm * num_sms(); }

struct ChunkInfo {   // per chunk, computed by k_prep_chunks
  int64_t cb0;       // first block (snapped to a window start in mode 0)
  int32_t wl;        // first window with RowWindowOffset[w] >= cb0 (nwin if none)
  int32_t pad;
};

struct Params {
  CUtensorMap cmap;          // C [M x N] fp32, box 32 columns x window height (TMA stores)
  const int32_t* rwo;        // RowWindowOffset [nwin+1]
  const uint8_t* tile;       // TCblocktileId [nnz]
  const int32_t* toff;       // TCblockoffset [T+1]
  const int32_t* s2x;        // SparseAToX [T*W], 16-byte aligned
  const float* vals;         // tile-order values or null (A = 1)
  const float* B;            // [M x N] fp32 (tf32 form) / hi or q plane (split forms)
  const void* B1;            // second plane (split forms): ext bytes or fp8 row scales
  int32_t bformat;
  float* C;                  // [M x N]
  float* part;               // partial tiles [2*G x H x N] (balance mode)
  uint32_t* err;
  uint32_t* counter;         // [slices] chunk queue (null: one chunk per CTA)
  const ChunkInfo* chunks;   // [G+1] or null (the producer searches RowWindowOffset)
  uint64_t* stamps;          // per-CTA timer records or null (see record_cta_time)
  int32_t stamp_cap;
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

// Per-stage metadata (one ring slot). toff holds nb + 1 offsets; s2x the
// gathered row of every slot of the stage's blocks (zero past nb).
struct alignas(16) StageMeta {
  int64_t sb;          // first TC block of the stage
  int32_t nb;          // blocks in the stage; -1 marks the end of the CTA's work
  int32_t pad;
  int32_t toff[8];
  int32_t s2x[32];
};

enum : int32_t { kRecHead = 1, kRecTail = 2, kRecEmpty = 4, kRecEnd = 8, kRecPad = 16 };

// One row window as a CTA meets it inside a chunk.
struct alignas(16) WinRec {
  int64_t wb0, wb1;    // the window's blocks inside the chunk
  int64_t cb0, cb1;    // the chunk's blocks
  int64_t stage_base;  // this CTA's global stage index of the chunk's first stage
  int32_t w;           // window id
  int32_t chunk;       // chunk id
  int32_t flags;       // kRecHead: started before the chunk; kRecTail: continues after it
  int32_t pad;
};

__device__ __forceinline__ int32_t lower_bound_i32(const int32_t* a, int32_t n, int64_t x) {
  int32_t lo = 0, hi = n;
  while (lo < hi) {
    int32_t mid = (lo + hi) >> 1;
    if ((int64_t)__ldg(a + mid) < x) lo = mid + 1; else hi = mid;
  }
  return lo;
}

// The first index in [0, n) with a[i] >= x (n if none), searched 32-ary by a
// whole warp: one round of 32 parallel probes per factor of 32.
__device__ __forceinline__ int32_t warp_lower_bound(const int32_t* a, int32_t n, int64_t x,
                                                    int lane) {
  int32_t lo = 0, hi = n;  // the answer lies in [lo, hi]
  while (lo < hi) {
    const int32_t step = (hi - lo + 31) / 32;
    const int32_t pi = lo + lane * step;
    const bool ge = (pi < hi) ? ((int64_t)__ldg(a + pi) >= x) : true;
    const uint32_t m = __ballot_sync(0xffffffffu, ge);
    const int j = m ? __ffs(m) - 1 : 32;  // no lane: the answer lies past the last probe
    const int32_t nhi = min(lo + j * step, hi);
    lo = j > 0 ? lo + (j - 1) * step + 1 : lo;
    hi = nhi;
  }
  return lo;
}

// Chunk k's block range.
__device__ __forceinline__ void chunk_bounds(const Params& p, int32_t k, int lane, int64_t& c0,
                                             int64_t& c1) {
  c0 = (int64_t)k * p.T / p.G;
  c1 = (int64_t)(k + 1) * p.T / p.G;
  if (p.mode == 0) {  // snap to window starts: windows never split
    const int32_t w0 = warp_lower_bound(p.rwo, p.nwin, c0, lane);
    c0 = (w0 < p.nwin) ? __ldg(p.rwo + w0) : p.T;
    if (k + 1 < p.G) {
      const int32_t w1 = warp_lower_bound(p.rwo, p.nwin, c1, lane);
      c1 = (w1 < p.nwin) ? __ldg(p.rwo + w1) : p.T;
    } else {
      c1 = p.T;
    }
  }
}

// Fills the chunk table and resets the queue counters: one warp per chunk.
__global__ void k_prep_chunks(const Params p, ChunkInfo* info, uint32_t* counter, int slices) {
  const int lane = threadIdx.x & 31;
  const int32_t k = (int32_t)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
  if (k == 0)
    for (int i = lane; i < slices; i += 32) counter[i] = 0;
  if (k > p.G) return;
  int64_t c0, c1;
  if (k < p.G) {
    chunk_bounds(p, k, lane, c0, c1);
  } else {
    c0 = p.T;
  }
  const int32_t wl = warp_lower_bound(p.rwo, p.nwin, c0, lane);
  if (lane == 0) {
    info[k].cb0 = c0;
    info[k].wl = wl;
    info[k].pad = 0;
  }
}

// Optional per-CTA timer record: [entry, exit, smid, chunks] (globaltimer ns).
__device__ __forceinline__ void record_cta_time(const Params& p, int slot, uint64_t value) {
  const int c = blockIdx.x + gridDim.x * blockIdx.y;
  if (p.stamps && c < p.stamp_cap) p.stamps[4 * (size_t)c + slot] = value;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t dst, const void* src, uint32_t src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src),
               "r"(src_bytes)
               : "memory");
}
// Waits until every cp.async this thread issued has completed (before a role
// exits, so no copy is still writing shared memory when the CTA ends).
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}
__device__ __forceinline__ void cp_async_arrive_noinc(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Barrier wait by a whole warp; false (and the abort flag set) if any lane gave up.
__device__ __forceinline__ bool warp_wait(uint64_t* bar, uint32_t parity, uint32_t* err,
                                          volatile uint32_t* abort_flag) {
  const bool got = mbar_wait(bar, parity, err);
  if (!__all_sync(0xffffffffu, got) || *abort_flag) {
    *abort_flag = 1;
    return false;
  }
  return true;
}

// Shared-memory rings of the producer and the barriers guarding them.
struct SchedRings {
  StageMeta* meta;       // [kMetaDepth]
  uint64_t* meta_full;   // [kMetaDepth] 32 cp.async arrivals + 1 (producer lane 0)
  uint64_t* meta_empty;  // [kMetaDepth] one arrival per consuming role
  WinRec* rec;           // [kRecDepth]
  uint64_t* rec_full;    // [kRecDepth] 1 (producer lane 0)
  uint64_t* rec_empty;   // [kRecDepth] one arrival per epilogue warp and UMMA issuer
};

constexpr int kSchedBytes = kMetaDepth * (int)sizeof(StageMeta) + kRecDepth * (int)sizeof(WinRec) +
                            (2 * kMetaDepth + 2 * kRecDepth) * 8;

__device__ __forceinline__ SchedRings carve_rings(uint8_t* base) {
  SchedRings r;
  r.meta = reinterpret_cast<StageMeta*>(base);
  r.rec = reinterpret_cast<WinRec*>(base + kMetaDepth * sizeof(StageMeta));
  uint64_t* b = reinterpret_cast<uint64_t*>(base + kMetaDepth * sizeof(StageMeta) +
                                            kRecDepth * sizeof(WinRec));
  r.meta_full = b;
  r.meta_empty = b + kMetaDepth;
  r.rec_full = b + 2 * kMetaDepth;
  r.rec_empty = b + 2 * kMetaDepth + kRecDepth;
  return r;
}

__device__ __forceinline__ void init_rings(const SchedRings& r, uint32_t meta_consumers,
                                           uint32_t rec_consumers) {
  for (int i = 0; i < kMetaDepth; ++i) {
    mbar_init(&r.meta_full[i], 32 + 1);
    mbar_init(&r.meta_empty[i], meta_consumers);
  }
  for (int i = 0; i < kRecDepth; ++i) {
    mbar_init(&r.rec_full[i], 1);
    mbar_init(&r.rec_empty[i], rec_consumers);
  }
}

// The producer warp (all 32 lanes). Emits, for every chunk this CTA takes,
// its stages (P blocks of width BW each) and its window records, then
// kEndStages end stages and one end record.
template <int P, int BW, int ALIGN>
__device__ void produce(const Params& p, const SchedRings& r, int lane,
                        volatile uint32_t* abort_flag) {
  uint64_t gst = 0;   // stages emitted
  uint32_t rq = 0;    // records emitted
  bool ok = true;
  uint32_t* const ctr = p.counter ? p.counter + blockIdx.y : nullptr;
  auto claim = [&]() -> int32_t {
    int32_t k = 0;
    if (lane == 0) k = (int32_t)atomicAdd(ctr, 1u);
    return __shfl_sync(0xffffffffu, k, 0);
  };
  int64_t rec_cb1 = 0;  // end block of the chunk being walked
  auto emit_rec = [&](int32_t w, int64_t wb0, int64_t wb1, int64_t cb0, int64_t sbase,
                      int32_t chunk, int32_t flags) {
    if (!ok) return;
    const int s = (int)(rq % kRecDepth);
    if (!warp_wait(&r.rec_empty[s], ((rq / kRecDepth) & 1) ^ 1, p.err, abort_flag)) {
      ok = false;
      return;
    }
    if (lane == 0) {
      WinRec& x = r.rec[s];
      x.wb0 = wb0; x.wb1 = wb1; x.cb0 = cb0; x.cb1 = rec_cb1; x.stage_base = (int64_t)sbase;
      x.w = w; x.chunk = chunk; x.flags = flags; x.pad = 0;
      mbar_arrive(&r.rec_full[s]);
    }
    __syncwarp();
    ++rq;
  };
  // Metadata of cnt <= kEmitBatch consecutive stages into ring slots gst ..
  // gst + cnt - 1: stage i covers blocks [sb0 + i P, min(sb0 + (i+1) P, cb1))
  // (nb0 >= 0 overrides the block count of a single stage: the pad stage).
  // One pass of the warp per batch: lane i waits on slot i, every lane issues
  // at most one copy of each kind, then arrives once on each slot.
  auto emit_stages = [&](int64_t sb0, int cnt, int64_t cb1, int nb0) -> bool {
    auto nb_of = [&](int i) -> int {
      if (nb0 >= 0) return nb0;
      const int64_t sb = sb0 + (int64_t)i * P;
      return (int)((cb1 - sb) < P ? (cb1 - sb) : P);
    };
    bool got = true;
    if (lane < cnt) {
      const uint64_t g = gst + (uint64_t)lane;
      got = mbar_wait(&r.meta_empty[g % kMetaDepth], (uint32_t)((g / kMetaDepth) & 1) ^ 1, p.err);
    }
    if (!__all_sync(0xffffffffu, got) || *abort_flag) {
      *abort_flag = 1;
      ok = false;
      return false;
    }
    {  // SparseAToX: 8 lanes x 16 bytes per stage, zero past the stage's blocks
      const int i = lane >> 3, c = lane & 7;
      if (i < cnt) {
        const int nb = nb_of(i);
        const int64_t sb = sb0 + (int64_t)i * P;
        const bool v = 4 * c < nb * BW;
        cp_async16(smem_u32(&r.meta[(gst + i) % kMetaDepth].s2x[4 * c]),
                   p.s2x + (v ? sb * BW + 4 * c : 0), v ? 16u : 0u);
      }
    }
    {  // TCblockoffset[sb .. sb + nb]: P + 1 lanes per stage
      const int i = lane / (P + 1), c = lane - i * (P + 1);
      if (i < cnt) {
        const int nb = nb_of(i);
        const int64_t sb = sb0 + (int64_t)i * P;
        const bool v = c <= nb;
        cp_async4(smem_u32(&r.meta[(gst + i) % kMetaDepth].toff[c]), p.toff + (v ? sb + c : 0),
                  v ? 4u : 0u);
      }
    }
    for (int i = 0; i < cnt; ++i) cp_async_arrive_noinc(&r.meta_full[(gst + i) % kMetaDepth]);
    if (lane < cnt) {
      StageMeta& m = r.meta[(gst + lane) % kMetaDepth];
      m.sb = sb0 + (int64_t)lane * P;
      m.nb = nb_of(lane);
      mbar_arrive(&r.meta_full[(gst + lane) % kMetaDepth]);
    }
    __syncwarp();
    gst += (uint64_t)cnt;
    return true;
  };
  // RowWindowOffset cursor: lane i holds rwo[wb + i] (entries past nwin read as
  // T + 1); the next batch (wb + 31 ...) is loaded one batch ahead.
  int32_t wb = 0;
  int64_t rv = 0, rv_next = 0;
  auto ld = [&](int32_t w) -> int64_t {
    return (w <= p.nwin) ? (int64_t)__ldg(p.rwo + w) : p.T + 1;
  };
  auto load_batch = [&](int32_t w) {
    wb = w;
    rv = ld(wb + lane);
    rv_next = ld(wb + 31 + lane);
  };
  auto rwo_at = [&](int32_t w) -> int64_t {  // w in [wb, wb + 31]
    return __shfl_sync(0xffffffffu, rv, w - wb);
  };
  // the last window w >= wb with rwo[w] <= b (the nonempty window holding block
  // b when b < T); on return the batch holds both w and w + 1
  auto last_le = [&](int64_t b) -> int32_t {
    while (true) {
      const int c = __popc(__ballot_sync(0xffffffffu, rv <= b));
      if (c < 32) return wb + c - 1;
      wb += 31;  // the preloaded batch starts at the old lane 31
      rv = rv_next;
      rv_next = ld(wb + 31 + lane);
    }
  };
  const int32_t first = ctr ? claim() : (int32_t)blockIdx.x;
  int32_t next = (!ctr || first >= p.G) ? p.G : claim();
  int32_t k = first;
  int64_t nc0 = 0, nc1 = 0;
  int32_t nwl = 0;
  auto info = [&](int32_t kk, int64_t& c0, int64_t& c1, int32_t& wl) {
    if (p.chunks) {
      c0 = __ldg(&p.chunks[kk].cb0);
      c1 = __ldg(&p.chunks[kk + 1].cb0);
      wl = __ldg(&p.chunks[kk].wl);
    } else {
      chunk_bounds(p, kk, lane, c0, c1);
      wl = warp_lower_bound(p.rwo, p.nwin, c0, lane);
    }
  };
  if (k < p.G) info(k, nc0, nc1, nwl);
  int chunks_done = 0;
  while (ok && k < p.G) {
    const int64_t cb0 = nc0, cb1 = nc1;
    const int32_t wl = nwl;
    const int32_t kc = k;
    // look up the next chunk now, so its loads overlap this chunk's stages
    k = next;
    if (k < p.G) {
      info(k, nc0, nc1, nwl);
      next = ctr ? claim() : p.G;
    }
    ++chunks_done;
    const bool last_chunk = (kc == p.G - 1);
    if (cb0 >= cb1 && !last_chunk) continue;
    rec_cb1 = cb1;
    while (ok && (gst % ALIGN) != 0 && cb0 < cb1) {  // pad stages: align the chunk's start
      const int64_t pad_stage = (int64_t)gst;
      if (!emit_stages(cb0, 1, cb1, 0)) break;
      emit_rec(-1, cb0, cb0, cb0, pad_stage, kc, kRecPad);
    }
    if (!ok) break;
    const int64_t sbase = (int64_t)gst;
    int32_t wcur = -1;     // current nonempty window
    int64_t wend = cb0;    // its end (block)
    load_batch(wl > 0 ? wl - 1 : 0);
    if (cb0 < cb1) {
      // windows starting at cb0 that are empty, then the one holding block cb0
      const bool at_start = wl < p.nwin && rwo_at(wl) == cb0;
      const int32_t w = last_le(cb0);
      const int32_t wfirst = at_start ? wl : w;
      for (int32_t e = wfirst; e < w; ++e) emit_rec(e, cb0, cb0, cb0, sbase, kc, kRecEmpty);
      const int64_t r0 = rwo_at(w), r1 = rwo_at(w + 1);
      emit_rec(w, r0 > cb0 ? r0 : cb0, r1 < cb1 ? r1 : cb1, cb0, sbase, kc,
               (r0 < cb0 ? kRecHead : 0) | (r1 > cb1 ? kRecTail : 0));
      wcur = w;
      wend = r1;
    }
    const int64_t nst = (cb1 - cb0 + P - 1) / P;
    for (int64_t j = 0; j < nst && ok;) {
      const int cnt = (int)((nst - j) < kEmitBatch ? (nst - j) : kEmitBatch);
      if (!emit_stages(cb0 + j * P, cnt, cb1, -1)) break;
      j += cnt;
      const int64_t send = (cb0 + j * P) < cb1 ? (cb0 + j * P) : cb1;
      // windows that start inside these stages
      while (ok && wend < send) {
        const int32_t w = last_le(wend);
        for (int32_t e = wcur + 1; e < w; ++e) emit_rec(e, wend, wend, cb0, sbase, kc, kRecEmpty);
        const int64_t r1 = rwo_at(w + 1);
        emit_rec(w, wend, r1 < cb1 ? r1 : cb1, cb0, sbase, kc, r1 > cb1 ? kRecTail : 0);
        wcur = w;
        wend = r1;
      }
    }
    if (ok && last_chunk) {  // empty windows after the last block belong to the last chunk
      const int32_t wl_end = (cb0 < cb1) ? wcur + 1 : wl;
      for (int32_t e = wl_end; e < p.nwin; ++e) emit_rec(e, p.T, p.T, cb0, sbase, kc, kRecEmpty);
    }
  }
  if (!ok) {
    *abort_flag = 1;
    cp_async_wait_all();
    return;
  }
  // end markers
  for (int i = 0; i < kEndStages; ++i, ++gst) {
    const int s = (int)(gst % kMetaDepth);
    if (!warp_wait(&r.meta_empty[s], (uint32_t)((gst / kMetaDepth) & 1) ^ 1, p.err,
                   abort_flag)) {
      cp_async_wait_all();
      return;
    }
    if (lane == 0) r.meta[s].nb = -1;
    __syncwarp();
    mbar_arrive(&r.meta_full[s]);  // 32 lanes
    if (lane == 0) mbar_arrive(&r.meta_full[s]);
    __syncwarp();
  }
  emit_rec(-1, 0, 0, 0, 0, -1, kRecEnd);
  cp_async_wait_all();
  if (lane == 0) record_cta_time(p, 3, (uint64_t)chunks_done);
}

// Byte offset of A_b^T element (window row r, slot s) in the K-major,
// no-swizzle core-matrix layout (8 rows x 16 B core matrices; LBO = 128 B
// between the two K halves, SBO = 256 B between the two 8-row groups).
__device__ __forceinline__ uint32_t y_offset(uint32_t pos) {
  uint32_t r = pos >> 3, s = pos & 7;
  return (r & 7) * 16 + (r >> 3) * 256 + (s >> 2) * 128 + (s & 3) * 4;
}

// Sums the partial tiles of every window cut by chunk boundaries, in chunk
// order (bitwise reproducible), and writes its C rows. One CTA per boundary.
__global__ void k_reduce_partials(const Params p) {
  const int c = blockIdx.x + 1;  // boundary between chunk c-1 and c
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
  // contributors: chunk c-1 (tail slot), chunks c..c_last (head slots)
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

// Writes the epilogue of 0 into the C rows of an empty window (columns of this
// CTA's slice, `nthreads` threads starting at thread t).
__device__ __forceinline__ void zero_window_rows(const Params& p, int32_t w, int col0, int ncols,
                                                 int t, int nthreads) {
  const int64_t row0 = (int64_t)w * p.H;
  for (int f = col0 + t; f < col0 + ncols; f += nthreads)
    for (int r = 0; r < p.H && row0 + r < p.M; ++r) p.C[(row0 + r) * p.N + f] = epilogue(p, 0.0f, f);
}

// Bytes of the chunk table for G chunks (the queue region is kQueueHeader of
// counters followed by the table).
inline size_t chunk_table_bytes(int G) {
  return align_up((size_t)(G + 1) * sizeof(ChunkInfo), 256);
}

// CTAs per N-slice: one per SM when the chunk queue is set up (persistent),
// else one per chunk.
inline int launch_ctas(const Params& p, int slices) {
  if (!p.counter) return p.G;
  int per = num_sms() / slices;
  if (per < 1) per = 1;
  return per < p.G ? per : p.G;
}

// Points the kernel at the queue region of the caller's workspace (counters +
// chunk table, 256-byte aligned) and launches k_prep_chunks to fill it; with
// no region the kernel runs one CTA per chunk.
inline dtc_status setup_queue(Params& p, void* queue, int slices, cudaStream_t st) {
  p.counter = nullptr;
  p.chunks = nullptr;
  p.stamps = cta_timer_buffer(&p.stamp_cap);
  if (!queue) return DTC_OK;
  DTC_REQUIRE(((uintptr_t)queue & 255) == 0, "queue region must be 256-byte aligned");
  DTC_REQUIRE((size_t)slices * 4 <= kQueueHeader, "too many N-slices for the chunk queue");
  p.counter = reinterpret_cast<uint32_t*>(queue);
  ChunkInfo* info = reinterpret_cast<ChunkInfo*>(reinterpret_cast<char*>(queue) + kQueueHeader);
  p.chunks = info;
  const int threads = 256;
  const int64_t warps = (int64_t)p.G + 1;
  const unsigned blocks = (unsigned)((warps * 32 + threads - 1) / threads);
  k_prep_chunks<<<blocks, threads, 0, st>>>(p, info, p.counter, slices);
  DTC_CUDA(cudaGetLastError());
  return DTC_OK;
}

}  // namespace
}  // namespace dtc
