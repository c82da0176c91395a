/*
 * ORACLE -- test infrastructure only.  Nothing in the product links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only as the checker (or the timed CPU baseline).
 *
 * CPU restatement of the reference DTC-SpMM ME-TCF conversion and a CSR SpMM
 * oracle. Every function cites the reference lines it follows (paths relative
 * to the reference project root).
 *
 *   ME-TCF conversion ........ DTC-SpMM/DTCSpMM_kernel.cu:107-419,
 *                              DTC-SpMM/DTCSpMM.cpp:313-359
 *   implicit A = 1 semantics . DTC-SpMM/DTCSpMM_kernel.cu:837-838, 2700-2703
 *                              (tile entries are *assigned*, so duplicate
 *                              (row, col) pairs collapse to one 1.0)
 *
 * Pinned against golden vectors produced by the reference's own conversion
 * (tests/golden/, generated by tests/golden/make_golden.py).
 *
 * Build: oracle/build_oracle.py -> oracle/_build/libmetcf_oracle.so
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int cmp_i32(const void* a, const void* b) {
  int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

/* Sorted distinct column ids of one row window.
 * DTCSpMM_kernel.cu:350-362 (sort of (window, col) pairs) and :176-187
 * (in-place deduplication). Returns |U_w|; *out is malloc'ed. */
static int32_t window_unique(const int32_t* col, int64_t e0, int64_t e1, int32_t** out) {
  int64_t n = e1 - e0;
  int32_t* u = (int32_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
  if (n > 0) memcpy(u, col + e0, (size_t)n * sizeof(int32_t));
  qsort(u, (size_t)n, sizeof(int32_t), cmp_i32);
  int64_t loc = 0;
  for (int64_t i = 1; i < n; i++)
    if (u[i] != u[loc]) u[++loc] = u[i];
  *out = u;
  return n > 0 ? (int32_t)(loc + 1) : 0;
}

/* First index of `key` in sorted distinct array u[0..n); -1 if absent.
 * DTCSpMM_kernel.cu:159-175 (binarysearch returns the first occurrence). */
static int32_t rank_of(const int32_t* u, int32_t n, int32_t key) {
  int32_t lo = 0, hi = n - 1;
  while (lo <= hi) {
    int32_t mid = lo + (hi - lo) / 2;
    if (u[mid] == key) return mid;
    if (u[mid] < key) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

/* Number of TC blocks T of the conversion (sum of blockPartition).
 * DTCSpMM_kernel.cu:205-228: blockPartition[w] = (last_idx + W) / W = ceil(|U_w|/W);
 * empty windows keep the caller's 0. */
int64_t oracle_metcf_num_blocks(const int32_t* rowptr, const int32_t* col,
                                int32_t M, int32_t H, int32_t W) {
  int32_t nwin = (M + H - 1) / H;
  int64_t T = 0;
  for (int32_t w = 0; w < nwin; w++) {
    int64_t e0 = rowptr[(int64_t)w * H];
    int64_t r1 = (int64_t)w * H + H; if (r1 > M) r1 = M;
    int64_t e1 = rowptr[r1];
    int32_t* u; int32_t nu = window_unique(col, e0, e1, &u);
    T += (nu + W - 1) / W;
    free(u);
  }
  return T;
}

/* Full ME-TCF conversion with the reference's exact output semantics.
 *  edgeToRow[e]         = row of e                        (:107-120)
 *  blockPartition[w]    = ceil(|U_w| / W), 0 if empty      (:205-228)
 *  edgeToColumn[e]      = rank of col(e) in U_w            (:224-227)
 *  RowWindowOffset      = [0, inclusive_scan(blockPartition)]  (:366-373)
 *  TCblockRowid[b]      = window of block b                (:149-173)
 *  TCblockoffset        = [0, inclusive_scan(nnz per block)]   (:270-280, :399-403)
 *  TCblocktileId        = (row % H) * W + rank % W, u8, stored per block in
 *                         CSR edge order                  (:287-300)
 *  SparseAToX[b*W + s]  = original column of slot s, 0 where unused (:296, :390-391)
 * All output arrays must be sized by the caller (T from oracle_metcf_num_blocks). */
int oracle_metcf(const int32_t* rowptr, const int32_t* col, int32_t M, int32_t H, int32_t W,
                 int32_t* blockPartition, int32_t* edgeToColumn, int32_t* edgeToRow,
                 int32_t* rowWindowOffset, int32_t* tcblockRowid, uint8_t* tileId,
                 int32_t* tcblockOffset, int32_t* sparseAToX, int64_t T) {
  int32_t nwin = (M + H - 1) / H;
  for (int32_t r = 0; r < M; r++)
    for (int64_t e = rowptr[r]; e < rowptr[r + 1]; e++) edgeToRow[e] = r;
  memset(sparseAToX, 0, (size_t)T * W * sizeof(int32_t));
  rowWindowOffset[0] = 0;
  tcblockOffset[0] = 0;
  int64_t b_base = 0;
  int32_t* cnt = NULL; int32_t* pos = NULL; int64_t cap = 0;
  for (int32_t w = 0; w < nwin; w++) {
    int64_t e0 = rowptr[(int64_t)w * H];
    int64_t r1 = (int64_t)w * H + H; if (r1 > M) r1 = M;
    int64_t e1 = rowptr[r1];
    int32_t* u; int32_t nu = window_unique(col, e0, e1, &u);
    int32_t nb = (nu + W - 1) / W;
    blockPartition[w] = nb;
    rowWindowOffset[w + 1] = (int32_t)(b_base + nb);
    if (b_base + nb > T) { free(u); free(cnt); free(pos); return -1; }
    for (int32_t b = 0; b < nb; b++) tcblockRowid[b_base + b] = w;
    if (nb > cap) { cap = nb; cnt = realloc(cnt, cap * sizeof(int32_t)); pos = realloc(pos, cap * sizeof(int32_t)); }
    for (int32_t b = 0; b < nb; b++) { cnt[b] = 0; pos[b] = 0; }
    for (int64_t e = e0; e < e1; e++) {
      int32_t rk = rank_of(u, nu, col[e]);
      edgeToColumn[e] = rk;
      cnt[rk / W]++;
    }
    /* per-window exclusive offsets, global inclusive scan (:270-280, :399-403) */
    int64_t run = e0;
    for (int32_t b = 0; b < nb; b++) {
      tcblockOffset[b_base + b + 1] = (int32_t)(run + cnt[b]);
      pos[b] = (int32_t)(run - e0);
      run += cnt[b];
    }
    for (int64_t e = e0; e < e1; e++) {
      int32_t rk = edgeToColumn[e];
      int32_t b = rk / W, s = rk % W;
      tileId[e0 + pos[b]] = (uint8_t)((edgeToRow[e] % H) * W + s);
      pos[b]++;
      sparseAToX[(b_base + b) * W + s] = col[e];
    }
    free(u);
    b_base += nb;
  }
  free(cnt); free(pos);
  return b_base == T ? 0 : -2;
}

/* Values permuted into TC-block (tile) order, the array the reference lacks
 * (it hard-codes A = 1, DTCSpMM_kernel.cu:837-838). Duplicate (row, col)
 * entries of one block are merged deterministically: the first occurrence in
 * CSR order carries the fp32 sum in CSR order, later ones carry 0. */
int oracle_metcf_values(const int32_t* rowptr, const int32_t* col, const float* val,
                        int32_t M, int32_t H, int32_t W, const int32_t* edgeToColumn,
                        const int32_t* edgeToRow, const int32_t* rowWindowOffset,
                        const int32_t* tcblockOffset, float* tcValues) {
  (void)col;
  int32_t nwin = (M + H - 1) / H;
  for (int32_t w = 0; w < nwin; w++) {
    int64_t e0 = rowptr[(int64_t)w * H];
    int64_t r1 = (int64_t)w * H + H; if (r1 > M) r1 = M;
    int64_t e1 = rowptr[r1];
    int32_t b0 = rowWindowOffset[w], nb = rowWindowOffset[w + 1] - b0;
    if (nb == 0) continue;
    int64_t* first = (int64_t*)malloc((size_t)nb * H * W * sizeof(int64_t));
    int64_t* pos = (int64_t*)calloc((size_t)nb, sizeof(int64_t));
    for (int64_t i = 0; i < (int64_t)nb * H * W; i++) first[i] = -1;
    for (int64_t e = e0; e < e1; e++) {
      int32_t b = edgeToColumn[e] / W;
      int64_t o = tcblockOffset[b0 + b] + pos[b]++;
      int64_t p = (int64_t)b * H * W + (edgeToRow[e] % H) * W + edgeToColumn[e] % W;
      if (first[p] < 0) { first[p] = o; tcValues[o] = val[e]; }
      else { tcValues[first[p]] += val[e]; tcValues[o] = 0.0f; }
    }
    free(first); free(pos);
  }
  return 0;
}

/* FP64 CSR SpMM oracle: C[i, :] = sum_e A[i, col_e] * B[col_e, :].
 * val == NULL reproduces the reference's implicit A = 1 with tile assignment
 * (duplicate (row, col) pairs count once); otherwise duplicates are summed. */
void oracle_spmm_f64(const int32_t* rowptr, const int32_t* col, const float* val,
                     int32_t M, int32_t N, const float* B, double* C) {
  #pragma omp parallel for schedule(dynamic, 64)
  for (int32_t i = 0; i < M; i++) {
    double* c = C + (int64_t)i * N;
    for (int32_t j = 0; j < N; j++) c[j] = 0.0;
    int64_t e0 = rowptr[i], e1 = rowptr[i + 1];
    for (int64_t e = e0; e < e1; e++) {
      if (!val) {
        int dup = 0;
        for (int64_t f = e0; f < e; f++) if (col[f] == col[e]) { dup = 1; break; }
        if (dup) continue;
      }
      double a = val ? (double)val[e] : 1.0;
      const float* b = B + (int64_t)col[e] * N;
      for (int32_t j = 0; j < N; j++) c[j] += a * (double)b[j];
    }
  }
}

/* Per-element magnitude bound sum_e |A[i,col_e]| * |B[col_e, j]| (FP64), used
 * by tests to scale the error tolerance of each output element. */
void oracle_spmm_absbound_f64(const int32_t* rowptr, const int32_t* col, const float* val,
                              int32_t M, int32_t N, const float* B, double* C) {
  #pragma omp parallel for schedule(dynamic, 64)
  for (int32_t i = 0; i < M; i++) {
    double* c = C + (int64_t)i * N;
    for (int32_t j = 0; j < N; j++) c[j] = 0.0;
    for (int64_t e = rowptr[i]; e < rowptr[i + 1]; e++) {
      double a = val ? fabs((double)val[e]) : 1.0;
      const float* b = B + (int64_t)col[e] * N;
      for (int32_t j = 0; j < N; j++) c[j] += a * fabs((double)b[j]);
    }
  }
}

/* Host CSR SpMM in FP32, row-parallel over `nthreads` OpenMP threads and
 * vectorised over N: the CPU baseline the benchmark times. */
void oracle_spmm_f32(const int32_t* rowptr, const int32_t* col, const float* val,
                     int32_t M, int32_t N, const float* B, float* C, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
  #pragma omp parallel for schedule(dynamic, 256)
  for (int32_t i = 0; i < M; i++) {
    float* c = C + (int64_t)i * N;
    for (int32_t j = 0; j < N; j++) c[j] = 0.0f;
    for (int64_t e = rowptr[i]; e < rowptr[i + 1]; e++) {
      float a = val ? val[e] : 1.0f;
      const float* b = B + (int64_t)col[e] * N;
      #pragma omp simd
      for (int32_t j = 0; j < N; j++) c[j] += a * b[j];
    }
  }
}

/* C from the ME-TCF arrays directly, FP64: C[w*H + r, :] += tile[r][s] * B[SparseAToX[b*W+s], :].
 * tcValues == NULL: tile entries are assigned 1.0 (reference kernels,
 * DTCSpMM_kernel.cu:2700-2703); else tile entries accumulate tcValues. */
void oracle_metcf_spmm_f64(const int32_t* rowWindowOffset, const uint8_t* tileId,
                           const int32_t* tcblockOffset, const int32_t* sparseAToX,
                           const float* tcValues, int32_t M, int32_t H, int32_t W,
                           int32_t N, const float* B, double* C) {
  int32_t nwin = (M + H - 1) / H;
  memset(C, 0, (size_t)M * N * sizeof(double));
  double* tile = (double*)malloc((size_t)H * W * sizeof(double));
  for (int32_t w = 0; w < nwin; w++) {
    for (int32_t b = rowWindowOffset[w]; b < rowWindowOffset[w + 1]; b++) {
      for (int i = 0; i < H * W; i++) tile[i] = 0.0;
      for (int64_t e = tcblockOffset[b]; e < tcblockOffset[b + 1]; e++) {
        if (tcValues) tile[tileId[e]] += (double)tcValues[e];
        else tile[tileId[e]] = 1.0;
      }
      for (int r = 0; r < H; r++) {
        int64_t row = (int64_t)w * H + r;
        if (row >= M) break;
        for (int s = 0; s < W; s++) {
          double a = tile[r * W + s];
          if (a == 0.0) continue;
          const float* bb = B + (int64_t)sparseAToX[(int64_t)b * W + s] * N;
          for (int32_t j = 0; j < N; j++) C[row * N + j] += a * (double)bb[j];
        }
      }
    }
  }
  free(tile);
}

/* ---------------------------------------------------------------------------
 * Dense-operand storage forms, restated from their definitions (the device
 * packers live in the product's formats.cu; these are the checkers).
 * ------------------------------------------------------------------------- */

/* fp32 rounded to nearest-even at 16 significant bits, split into the bf16
 * top half ("hi") and the next 8 mantissa bits ("ext"). NaN -> canonical
 * quiet NaN, +-Inf kept. */
void oracle_pack_split24(const float* B, int64_t n, uint16_t* hi, uint8_t* ext) {
  for (int64_t i = 0; i < n; i++) {
    uint32_t u;
    memcpy(&u, &B[i], 4);
    uint32_t e = (u >> 23) & 0xFF;
    uint32_t r;
    if (e == 0xFF) r = (u & 0x7FFFFF) ? 0x7FC00000u : u;
    else r = (u + 0x7Fu + ((u >> 8) & 1u)) & 0xFFFFFF00u;
    hi[i] = (uint16_t)(r >> 16);
    ext[i] = (uint8_t)(r >> 8);
  }
}

/* fp32 -> bf16, round to nearest even; NaN -> quiet NaN keeping the sign. */
void oracle_pack_bf16(const float* B, int64_t n, uint16_t* out) {
  for (int64_t i = 0; i < n; i++) {
    uint32_t u;
    memcpy(&u, &B[i], 4);
    if (((u >> 23) & 0xFF) == 0xFF && (u & 0x7FFFFF)) { out[i] = (uint16_t)((u >> 16) | 0x40); continue; }
    out[i] = (uint16_t)((u + 0x7FFFu + ((u >> 16) & 1u)) >> 16);
  }
}

/* fp32 -> e4m3 (1 sign, 4 exponent bits with bias 7, 3 mantissa bits; no
 * infinities, S.1111.111 is NaN, largest finite 448), round to nearest even,
 * saturating to +-448. */
static uint8_t e4m3_rn_sat(float y) {
  if (isnan(y)) return 0x7F;
  uint8_t sign = signbit(y) ? 0x80 : 0x00;
  double a = fabs((double)y);
  if (a >= 448.0) return sign | 0x7E;
  if (a < ldexp(1.0, -6)) {                 /* subnormal range: multiples of 2^-9 */
    double m = nearbyint(a * 512.0);        /* 0..8; 8 encodes the smallest normal */
    return sign | (uint8_t)m;
  }
  int e;
  frexp(a, &e);                             /* a = f * 2^e, f in [0.5, 1) */
  e -= 1;                                   /* a in [2^e, 2^(e+1)) */
  double t = nearbyint(ldexp(a, 3 - e));    /* 8..16 */
  if (t >= 16.0) { t = 8.0; e += 1; }
  if (e > 8 || (e == 8 && t > 14.0)) return sign | 0x7E;
  return sign | (uint8_t)(((e + 7) << 3) | ((int)t - 8));
}

/* Per-row scale s = max|B[r,:]| / 448 (1 when the row is all zero or not
 * finite), q = e4m3(B / s). */
void oracle_pack_fp8(const float* B, int64_t rows, int32_t N, uint8_t* q, float* scale) {
  for (int64_t r = 0; r < rows; r++) {
    const float* x = B + r * N;
    float m = 0.0f;
    for (int32_t j = 0; j < N; j++) { float v = fabsf(x[j]); if (v > m) m = v; }
    float s = (m > 0.0f && isfinite(m)) ? m / 448.0f : 1.0f;
    scale[r] = s;
    for (int32_t j = 0; j < N; j++) q[r * N + j] = e4m3_rn_sat(x[j] / s);
  }
}

/* Value of an e4m3 byte (for error bounds in tests). */
float oracle_e4m3_value(uint8_t b) {
  int s = b >> 7, e = (b >> 3) & 0xF, m = b & 7;
  if (e == 0xF && m == 7) return NAN;
  float v = e == 0 ? ldexpf((float)m, -9) : ldexpf(1.0f + m / 8.0f, e - 7);
  return s ? -v : v;
}
