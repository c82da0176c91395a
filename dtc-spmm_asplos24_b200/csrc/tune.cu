// Exhaustive schedule autotuner for the TC-block SpMM (dtc_autotune).
//
// The reference picks its schedule from a hand-written table per dataset and
// N (scripts/DTCSpMM/run_DTC_SpMM.py:10-30: balance or not, vector width,
// N split). Here the schedule knobs of the tcgen05 kernels are measured
// instead, on the caller's own ME-TCF arrays and B:
//   mode   0 = window-scheduled (windows never split), 1 = strict balance
//          (windows longer than the per-CTA chunk are split; the chunk,
//          ceil(T / grid) blocks, is the split threshold)
//   waves  chunks = waves x SMs, pulled by one persistent CTA per SM from a
//          device counter (more chunks even out skew at the price of more
//          chunk boundaries); window mode also tries 32 and 64, balance mode,
//          whose cut windows need partial tiles per chunk, stops at 16
//   ntile  128-feature tiles per CTA (fewer tiles spread wide N over more CTAs)
// Each candidate runs once untimed and `reps` times between CUDA events on the
// caller's stream; the mean is its time. Candidates change neither the B form
// nor the product precision, only how fp32 partial sums are grouped; each
// candidate's result is bitwise reproducible (window mode writes every C
// element once, balance mode reduces its partial tiles in fixed order).
#include <vector>
#include "impl.h"


using namespace dtc;

namespace {

constexpr int kWaveChoices[] = {1, 2, 4, 8, 16, 32, 64};
constexpr int kMaxWaves = 64;         // chunks of the queue region
constexpr int kMaxBalanceWaves = 16;  // chunks with partial tiles (balance mode)

// N-tiles per CTA when the caller does not cap them (see the kernels' dispatch).
int auto_ntile(int32_t N, int H, bool split) {
  const int nt = N <= 128 ? 1 : N <= 256 ? 2 : 4;
  return (split && H == 32 && nt > 2) ? 2 : nt;
}

// Every distinct (mode, waves, ntile) the kernels support for this N.
int candidates(int32_t N, int H, bool split, dtc_schedule* out, int max) {
  int n = 0;
  const int nt_auto = auto_ntile(N, H, split);
  for (int mode = 0; mode <= 1; ++mode)
    for (int w : kWaveChoices)
      for (int nt = 1; nt <= 4; nt *= 2) {
        if (mode == 1 && w > kMaxBalanceWaves) break;
        if (nt > nt_auto) break;
        if (out && n < max) {
          dtc_schedule& s = out[n];
          s.mode = mode;
          s.waves = w;
          s.ntile = nt;
          s.grid = 0;
          s.ms = 0.0f;
        }
        ++n;
      }
  return n;
}

struct Events {
  cudaEvent_t a = nullptr, b = nullptr;
  ~Events() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

}  // namespace

extern "C" {

int dtc_schedule_candidates(int32_t N, dtc_schedule* out, int max_out) {
  if (N < 1) return 0;
  return candidates(N, 16, false, out, max_out);
}

int dtc_schedule_candidates_ex(int32_t N, int32_t block_h, int split, dtc_schedule* out,
                               int max_out) {
  if (N < 1 || (block_h != 16 && block_h != 32)) return 0;
  return candidates(N, block_h, split != 0, out, max_out);
}

dtc_status dtc_autotune_workspace_bytes(int32_t num_nodes, int64_t num_blocks, int32_t N,
                                        int32_t block_h, size_t* bytes) {
  DTC_REQUIRE(bytes != nullptr, "bytes is null");
  DTC_REQUIRE(num_nodes >= 0 && num_blocks >= 0 && N >= 1, "bad sizes");
  DTC_REQUIRE(block_h == 16 || block_h == 32, "block_h must be 16 or 32");
  *bytes = align_up(spmm_partials_bytes(num_blocks, N, kMaxBalanceWaves * num_sms(), block_h), 256) +
           spmm_queue_bytes(num_blocks, kMaxWaves * num_sms());
  return DTC_OK;
}

dtc_status dtc_autotune(const int32_t* d_rowWindowOffset, const uint8_t* d_tileId,
                        const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                        const float* d_tcValues, int32_t num_nodes, int32_t num_windows,
                        int64_t num_blocks, int32_t block_h, int32_t block_w, int bformat,
                        const void* d_Bplane0,
                        const void* d_Bplane1, int32_t N, int precision, float* d_C,
                        void* d_workspace, size_t workspace_bytes, int reps,
                        dtc_schedule* results, int max_results, int* num_results, int* best,
                        dtc_stream_t stream) {
  DTC_REQUIRE(d_rowWindowOffset && d_tcblockOffset && d_Bplane0 && d_C, "null device pointer");
  DTC_REQUIRE(num_nodes >= 0 && num_blocks >= 0 && N >= 1, "bad sizes");
  DTC_REQUIRE(reps >= 1 && reps <= 1000, "reps must be in [1, 1000]");
  DTC_REQUIRE(best != nullptr, "best is null");
  size_t need = 0;
  dtc_status s = dtc_autotune_workspace_bytes(num_nodes, num_blocks, N, block_h, &need);
  if (s != DTC_OK) return s;
  if (!d_workspace || workspace_bytes < need) {
    set_error("autotune workspace too small (dtc_autotune_workspace_bytes)");
    return DTC_ERR_WORKSPACE_TOO_SMALL;
  }
  const bool tf32 = (bformat == DTC_B_F32 && precision == DTC_PREC_TF32);
  if (tf32) {
    DTC_REQUIRE(N % 4 == 0, "tcgen05 path needs N % 4 == 0");
  } else {
    DTC_REQUIRE(N % 16 == 0, "split-precision path needs N % 16 == 0");
  }
  const int ncand_all = candidates(N, block_h, !tf32, nullptr, 0);
  std::vector<dtc_schedule> cand(ncand_all);
  candidates(N, block_h, !tf32, cand.data(), ncand_all);
  if (!tf32 && block_w == 16) {  // the split kernels hold at most 2 N-tiles at width 16
    std::vector<dtc_schedule> kept;
    for (const dtc_schedule& c : cand)
      if (c.ntile <= 2) kept.push_back(c);
    cand.swap(kept);
  }
  const int ncand = (int)cand.size();
  cudaStream_t st = (cudaStream_t)stream;
  Events ev;
  DTC_CUDA(cudaEventCreate(&ev.a));
  DTC_CUDA(cudaEventCreate(&ev.b));
  const int sms = num_sms();
  // the chunk queue sits after the largest candidate's partial tiles
  void* queue = queue_region(
      d_workspace, workspace_bytes,
      align_up(spmm_partials_bytes(num_blocks, N, kMaxBalanceWaves * sms, block_h), 256), num_blocks,
      kMaxWaves * sms);
  int best_i = -1;
  for (int i = 0; i < ncand; ++i) {
    dtc_schedule& c = cand[i];
    int64_t g = (int64_t)c.waves * sms;
    if (g > num_blocks) g = num_blocks > 0 ? num_blocks : 1;
    c.grid = (int32_t)g;
    auto run = [&]() {
      return tf32 ? spmm_tf32_impl(d_rowWindowOffset, d_tileId, d_tcblockOffset, d_sparseAToX,
                                   d_tcValues, num_nodes, num_windows, num_blocks,
                                   (const float*)d_Bplane0, N, d_C, c.mode, c.grid,
                                   (float*)d_workspace, st, c.ntile, Epilogue{}, block_h, queue,
                                   block_w)
                  : spmm_split_impl(d_rowWindowOffset, d_tileId, d_tcblockOffset, d_sparseAToX,
                                    d_tcValues, num_nodes, num_windows, num_blocks, bformat,
                                    d_Bplane0, d_Bplane1, N, precision, d_C, c.mode, c.grid,
                                    (float*)d_workspace, st, c.ntile, Epilogue{}, block_h, queue,
                                    block_w);
    };
    s = run();  // warm-up
    if (s != DTC_OK) return s;
    DTC_CUDA(cudaEventRecord(ev.a, st));
    for (int r = 0; r < reps; ++r) {
      s = run();
      if (s != DTC_OK) return s;
    }
    DTC_CUDA(cudaEventRecord(ev.b, st));
    DTC_CUDA(cudaEventSynchronize(ev.b));
    float ms = 0.0f;
    DTC_CUDA(cudaEventElapsedTime(&ms, ev.a, ev.b));
    c.ms = ms / reps;
    if (best_i < 0 || c.ms < cand[best_i].ms) best_i = i;
  }
  if (results)
    for (int i = 0; i < ncand && i < max_results; ++i) results[i] = cand[i];
  if (num_results) *num_results = ncand;
  *best = best_i;
  return DTC_OK;
}

}  // extern "C"
