/*
 * dtc_spmm.h -- C ABI of the B200-native DTC-SpMM path (libdtcspmm.so).
 *
 * Plain pointers and sizes only; every pointer named d_* is device memory on
 * the current device, every call is asynchronous on `stream` unless stated,
 * and every call returns a dtc_status (never exits the process). The library
 * allocates no device memory: callers pass a workspace sized by the matching
 * *_workspace_bytes query. The tcgen05 SpMM entry points read B and write C
 * with 16-byte accesses and TMA stores: d_B / B planes and d_C must be 16-byte
 * aligned and N a multiple of 4 (16 for the split-precision forms); other N
 * go to the legacy-ISA kernel where an entry point says so. They also read
 * d_sparseAToX in 16-byte pieces: it must be 16-byte aligned.
 *
 * Workspaces of the SpMM entry points hold the partial tiles of strict balance
 * (required) followed by a small chunk-queue region (optional): with it, one
 * CTA per SM pulls chunks of TC blocks from a device counter; with only the
 * required bytes, the kernels run one CTA per chunk. The *_workspace_bytes
 * queries return the size with the queue (workspace base 256-byte aligned).
 *
 * Each entry point names the reference interface it replaces (paths relative
 * to the reference project root, HPMLL/DTC-SpMM_ASPLOS24).
 */
#ifndef DTC_SPMM_H_
#define DTC_SPMM_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef void* dtc_stream_t; /* a cudaStream_t; NULL = legacy default stream */

typedef enum {
  DTC_OK = 0,
  DTC_ERR_INVALID_ARGUMENT = 1,   /* bad size, null pointer, unsupported shape */
  DTC_ERR_WORKSPACE_TOO_SMALL = 2,
  DTC_ERR_CUDA = 3,               /* a CUDA runtime call failed; see dtc_last_error() */
  DTC_ERR_UNSUPPORTED = 4,        /* device or format not supported (e.g. not sm_100) */
  DTC_ERR_DEVICE_CHECK = 5        /* a kernel's own bounds / wait check fired */
} dtc_status;

/* Human-readable text of the last error recorded on the calling host thread. */
const char* dtc_last_error(void);

/* Library version (major*10000 + minor*100 + patch). */
int dtc_version(void);

/* Reads the device-side error word of the current device into *flags and
 * clears it if `clear` != 0 (synchronises the device). Bit 0: a bounded
 * in-kernel wait gave up; bit 1: an out-of-range index was skipped. No
 * reference counterpart (the reference has no device-side checks). */
dtc_status dtc_device_status(uint32_t* flags, int clear);

/* ------------------------------------------------------------------------- */
/* ME-TCF conversion.                                                         */
/* Replaces DTCSpMM.preprocess_gpu (DTC-SpMM/DTCSpMM.cpp:313-359) and its     */
/* launchers fill_edgeToRow_cuda / fill_segment_cuda / seg_sort_dequ          */
/* (DTC-SpMM/DTCSpMM_kernel.cu:107-419). Split in two phases because the      */
/* output sizes depend on the block count T (the reference reads T back to    */
/* the host at DTCSpMM_kernel.cu:378-380, so does dtc_convert_count).         */
/* ------------------------------------------------------------------------- */

/* Workspace for both conversion phases. */
dtc_status dtc_convert_workspace_bytes(int32_t num_nodes, int64_t nnz, int32_t block_h,
                                       int32_t block_w, size_t* bytes);

/* Phase 1. Inputs: CSR d_col[nnz] (edgeList), d_rowptr[num_nodes+1] (nodePointer).
 * Writes d_blockPartition[num_windows], d_edgeToColumn[nnz], d_edgeToRow[nnz]
 * (the reference's in-place outputs) and d_rowWindowOffset[num_windows+1];
 * stores T in *num_blocks (synchronises `stream`). block_h*block_w <= 256. */
dtc_status dtc_convert_count(const int32_t* d_col, const int32_t* d_rowptr, int32_t num_nodes,
                             int64_t nnz, int32_t block_h, int32_t block_w,
                             int32_t* d_blockPartition, int32_t* d_edgeToColumn,
                             int32_t* d_edgeToRow, int32_t* d_rowWindowOffset,
                             void* d_workspace, size_t workspace_bytes, int64_t* num_blocks,
                             dtc_stream_t stream);

/* Phase 2. Writes d_tcblockRowid[T], d_tileId[nnz] (u8), d_tcblockOffset[T+1],
 * d_sparseAToX[T*block_w]. If d_values (CSR order) is non-null, also writes
 * d_tcValues[nnz] in tile order (duplicate (row,col) pairs of a block merged
 * into their first occurrence, later ones 0) -- an array the reference lacks. */
dtc_status dtc_convert_fill(const int32_t* d_col, const int32_t* d_rowptr, int32_t num_nodes,
                            int64_t nnz, int32_t block_h, int32_t block_w,
                            const int32_t* d_edgeToColumn, const int32_t* d_edgeToRow,
                            const int32_t* d_rowWindowOffset, int64_t num_blocks,
                            int32_t* d_tcblockRowid, uint8_t* d_tileId, int32_t* d_tcblockOffset,
                            int32_t* d_sparseAToX, const float* d_values, float* d_tcValues,
                            void* d_workspace, size_t workspace_bytes, dtc_stream_t stream);

/* ------------------------------------------------------------------------- */
/* CSR relabelling. Output is canonical CSR: columns sorted within each row,  */
/* duplicate (row, col) entries merged by summing their values in input CSR  */
/* order (d_val == NULL counts each entry as 1, the reference's A = 1), the   */
/* number of output entries stored in *nnz_out (synchronises `stream`).       */
/* ------------------------------------------------------------------------- */
dtc_status dtc_relabel_workspace_bytes(int32_t num_rows, int32_t num_cols, int64_t nnz,
                                       size_t* bytes);

/* Symmetric permutation P A Pᵀ of a square matrix: output row i is input row
 * d_perm[i] with every column c renamed to the position of c in d_perm
 * (d_perm[new] = old, a permutation of [0, num_nodes)). Replaces the
 * reorder application of reordering/TCA_reorder.py:308-326 followed by the
 * CSR rebuild of scripts/DTCSpMM/dataset.py:38-44 (scipy coo -> csr).
 * d_val_out may be NULL. Output arrays hold num_nodes+1 / nnz entries. */
dtc_status dtc_permute_csr(const int32_t* d_rowptr, const int32_t* d_col, const float* d_val,
                           int32_t num_nodes, int64_t nnz, const int32_t* d_perm,
                           int32_t* d_rowptr_out, int32_t* d_col_out, float* d_val_out,
                           int64_t* nnz_out, void* d_workspace, size_t workspace_bytes,
                           dtc_stream_t stream);

/* Transpose: the num_cols x num_rows matrix Aᵀ, the operand of the backward
 * product Aᵀ·G. The reference has no transpose: its backward entry points
 * (DTC-SpMM/DTCSpMM.cpp:385-398) rerun the forward, valid only for symmetric
 * A. Output arrays hold num_cols+1 / nnz entries. */
dtc_status dtc_transpose_csr(const int32_t* d_rowptr, const int32_t* d_col, const float* d_val,
                             int32_t num_rows, int32_t num_cols, int64_t nnz,
                             int32_t* d_rowptr_out, int32_t* d_col_out, float* d_val_out,
                             int64_t* nnz_out, void* d_workspace, size_t workspace_bytes,
                             dtc_stream_t stream);

/* TCA reorder: two-level MinHash-LSH + Jaccard greedy clustering of rows
 * (reordering/TCA_reorder.py:53-326; its MinHash/LSH come from datasketch and
 * cuGraph, absent here, so hashing and banding are this library's own).
 * Writes d_perm[num_nodes] (d_perm[new] = old) for dtc_permute_csr. Row sets
 * are the distinct columns of each row of a square CSR matrix. Synchronises
 * `stream`; the merge loop runs on the host. Deterministic for given params. */
typedef struct {
  int32_t num_perm;       /* MinHash functions (reference: 128)                  */
  int32_t bands;          /* LSH bands; bands * rows_per_band <= num_perm        */
  int32_t rows_per_band;  /* (42 x 3 puts the LSH threshold near 0.2-0.3)        */
  int32_t thres;          /* level-1 cluster size cap in rows (reference: 16)    */
  int32_t c_thres;        /* level-2 cap in clusters (reference: 128)            */
  int32_t bucket_window;  /* each item pairs with this many bucket successors    */
  uint64_t seed;
} dtc_tca_params;

void dtc_tca_default_params(dtc_tca_params* params);
dtc_status dtc_tca_workspace_bytes(int32_t num_nodes, int64_t nnz, const dtc_tca_params* params,
                                   size_t* bytes);
dtc_status dtc_tca_reorder(const int32_t* d_rowptr, const int32_t* d_col, int32_t num_nodes,
                           int64_t nnz, const dtc_tca_params* params, int32_t* d_perm,
                           void* d_workspace, size_t workspace_bytes, dtc_stream_t stream);

/* One level of the TCA greedy merge on caller-given candidate pairs, in HOST
 * memory (no CUDA call): the merge loop of reordering/TCA_reorder.py:153-188
 * (level 1, cap `thres`) and :252-294 (level 2, cap `c_thres`), which
 * dtc_tca_reorder runs on its own LSH candidates. No counterpart entry in the
 * reference (its merge runs inline in the script); it lets a caller with
 * another candidate generator (for example datasketch's MinHash LSH) reuse the
 * merge. Items are num_items sets, CSR of sorted distinct members
 * (set_ptr[num_items+1], set_idx[set_ptr[num_items]]); pairs[num_pairs] are
 * lo << 32 | hi with lo < hi (duplicates ignored). Pairs pop by descending
 * Jaccard, equal scores in ascending (first, second) order; two roots merge,
 * the smaller cluster into the larger and equal sizes into the first member; a
 * cluster reaching `cap` is closed; a pair whose ends are not both roots is
 * requeued once as (root of first, root of second), keeping that orientation,
 * with the Jaccard of the two root items' own sets. Writes the
 * root of every item to roots[num_items]. Level 2 runs it again on the level-1
 * clusters (sets = the union of their rows' sets). */
dtc_status dtc_tca_merge(const int64_t* set_ptr, const int32_t* set_idx, int32_t num_items,
                         const uint64_t* pairs, int64_t num_pairs, int32_t cap, int32_t* roots);

/* COO edge list -> canonical CSR: the CSR build of the reference's loader
 * (scripts/DTCSpMM/dataset.py:21-44: src_li / dst_li / num_nodes of an .npz,
 * coo_matrix((1, (src, dst))).tocsr()). d_val == NULL gives every edge the
 * value 1, so duplicate edges sum to their multiplicity like the reference's.
 * Output arrays hold num_rows+1 / nnz entries. */
dtc_status dtc_coo_to_csr(const int32_t* d_src, const int32_t* d_dst, const float* d_val,
                          int32_t num_rows, int32_t num_cols, int64_t nnz, int32_t* d_rowptr_out,
                          int32_t* d_col_out, float* d_val_out, int64_t* nnz_out,
                          void* d_workspace, size_t workspace_bytes, dtc_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Dense-operand storage forms ("B formats").                                  */
/* ------------------------------------------------------------------------- */
typedef enum {
  DTC_B_F32 = 0,      /* fp32 rows; the TF32 drop-in form                      */
  DTC_B_SPLIT24 = 1,  /* bf16 hi plane [rows*N] + u8 extension plane [rows*N]: */
                      /* fp32 rounded to 16 significant bits, 3 bytes/element  */
  DTC_B_BF16 = 2,     /* bf16 rows                                              */
  DTC_B_FP8 = 3,      /* e4m3 plane [rows*N] + fp32 per-row scale [rows]        */
  DTC_B_BF16X2 = 4    /* bf16 hi plane + bf16 lo plane, lo = bf16(b - hi):      */
                      /* 4 bytes/element, ~16 significant bits, no rebuild      */
} dtc_bformat;

typedef enum {
  DTC_PREC_TF32 = 0,  /* tcgen05 kind::tf32, fp32 B                              */
  DTC_PREC_SPLIT3 = 1,/* kind::f16 bf16: A_hi*B_hi + A_hi*B_lo + A_lo*B_hi       */
  DTC_PREC_SPLIT4 = 2 /* kind::f16 bf16: (A_hi + A_lo) * (B_hi + B_lo), 4 terms  */
} dtc_precision;

/* Bytes of the two planes of `fmt` for a rows x N fp32 matrix. */
dtc_status dtc_bformat_bytes(int fmt, int64_t rows, int32_t N, size_t* plane0, size_t* plane1);

/* Converts fp32 d_B[rows*N] into `fmt` (plane1 unused for F32/BF16). */
dtc_status dtc_pack_b(int fmt, const float* d_B, int64_t rows, int32_t N, void* d_plane0,
                      void* d_plane1, dtc_stream_t stream);

/* ------------------------------------------------------------------------- */
/* TC-block SpMM  C[num_nodes x N] = A * B.                                    */
/* ------------------------------------------------------------------------- */

/* Window-scheduled SpMM. Replaces run_DTCSpMM / spmm_forward_ptx_uint8_improved
 * (DTC-SpMM/DTCSpMM.cpp:117-131 -> DTCSpMM_kernel.cu:811-944) and DTCSpMM_gcn
 * (DTCSpMM.cpp:147-161 -> DTCSpMM_kernel.cu:1033-1116): one launch, each row
 * window is owned by one CTA, no workspace. d_tcValues == NULL reproduces the
 * reference's implicit A = 1 (DTCSpMM_kernel.cu:837-838). C rows of empty
 * windows are written as zeros (the reference zero-fills, :823). */
dtc_status dtc_spmm(const int32_t* d_rowWindowOffset, const uint8_t* d_tileId,
                    const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                    const float* d_tcValues, int32_t num_nodes, int32_t num_windows,
                    int64_t num_blocks, const float* d_B, int32_t N, float* d_C,
                    dtc_stream_t stream);

/* Strict-balance SpMM. Replaces run_DTCSpMM_balance /
 * spmm_balance_forward_ptx_uint8_prefetch (DTC-SpMM/DTCSpMM.cpp:163-178 ->
 * DTCSpMM_kernel.cu:1118-1199, kernels :4730-4901, :5085-5362). Every CTA gets
 * an equal contiguous range of TC blocks (windows split across CTAs); partial
 * tiles go to the workspace and are reduced in fixed CTA order by a second
 * kernel, so results are bitwise reproducible (the reference uses fp32
 * atomicAdd). Needs only d_tcblockRowid, like the reference. */
dtc_status dtc_spmm_balance_workspace_bytes(int32_t num_nodes, int64_t num_blocks, int32_t N,
                                            size_t* bytes);
dtc_status dtc_spmm_balance(const int32_t* d_tcblockRowid, const uint8_t* d_tileId,
                            const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                            const float* d_tcValues, int32_t num_nodes, int64_t num_blocks,
                            const float* d_B, int32_t N, float* d_C, void* d_workspace,
                            size_t workspace_bytes, dtc_stream_t stream);

/* Strict-balance SpMM that allocates nothing and takes no workspace; no
 * counterpart in the reference. For callers that cannot call cudaMalloc
 * (a server whose device memory belongs to its own budgeted pool, plugins or
 * plain-C hosts without a device allocator): the window-offset table and the
 * partial tiles live in a fixed 16 MiB array compiled into the library, held
 * in the memory of every GPU that loads it until the process exits.
 * Limit: 4*(ceil(num_nodes/16)+1) bytes (rounded up to 256) + 128*N bytes per
 * SM (one CTA per SM) must fit in dtc_noalloc_scratch_capacity() bytes; larger
 * problems get DTC_ERR_WORKSPACE_TOO_SMALL. The first call on a device looks
 * up the array's device address with that device current -- make it before
 * any stream capture. All calls share the array: calls that overlap on the
 * GPU race and must be serialised by the caller. Same results semantics as
 * dtc_spmm_balance (deterministic for a given device). */
dtc_status dtc_spmm_balance_noalloc(const int32_t* d_tcblockRowid, const uint8_t* d_tileId,
                                    const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                                    const float* d_tcValues, int32_t num_nodes,
                                    int64_t num_blocks, const float* d_B, int32_t N, float* d_C,
                                    dtc_stream_t stream);
/* Bytes of the built-in scratch array used by dtc_spmm_balance_noalloc. */
size_t dtc_noalloc_scratch_capacity(void);

/* General form used by the tuned paths: any B format / precision, explicit
 * schedule. block_h x block_w = the ME-TCF's block shape (the conversion's
 * blockSize_h x blockSize_w, DTC-SpMM/DTCSpMM.cpp:315-316): 16 x 8, 32 x 8 or
 * 16 x 16 (the compaction width knob; tile ids must fit a byte).
 * mode 0 = window-scheduled, 1 = strict balance. grid = chunks G of the TC-block
 * range (0 = 16 per SM); the split threshold is ceil(num_blocks / G) blocks.
 * ntile = 128-feature tiles per CTA (0 = all of N up to 4, or up to 2 for the
 * split forms at block_h 32 or block_w 16; 1 or 2 split wider N across more
 * CTAs). d_rowWindowOffset is required (build it from TCblockRowid with
 * dtc_rowid_to_window_offset). Workspace: required in mode 1 (partial tiles),
 * optional chunk queue after it (see the top of this header). */
dtc_status dtc_spmm_ex(const int32_t* d_rowWindowOffset, const uint8_t* d_tileId,
                       const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                       const float* d_tcValues, int32_t num_nodes, int32_t num_windows,
                       int64_t num_blocks, int32_t block_h, int32_t block_w, int bformat,
                       const void* d_Bplane0, const void* d_Bplane1, int32_t N, int precision,
                       float* d_C, int mode, int grid, int ntile, void* d_workspace,
                       size_t workspace_bytes, dtc_stream_t stream);
dtc_status dtc_spmm_ex_workspace_bytes(int32_t num_nodes, int64_t num_blocks, int32_t N,
                                       int32_t block_h, int mode, int grid, size_t* bytes);

/* dtc_spmm_ex with the GCN layer's epilogue fused into the store of C:
 * C = act(A*B + bias), bias[N] per column (NULL = none), act = ReLU when
 * relu != 0. Replaces DTCSpMM_gcn (DTC-SpMM/DTCSpMM.cpp:147-161 ->
 * DTCSpMM_kernel.cu:1033-1116) followed by a separate bias/activation pass. */
dtc_status dtc_spmm_fused(const int32_t* d_rowWindowOffset, const uint8_t* d_tileId,
                          const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                          const float* d_tcValues, int32_t num_nodes, int32_t num_windows,
                          int64_t num_blocks, int32_t block_h, int32_t block_w, int bformat,
                          const void* d_Bplane0, const void* d_Bplane1, int32_t N, int precision,
                          const float* d_bias, int relu, float* d_C, int mode, int grid,
                          int ntile, void* d_workspace, size_t workspace_bytes,
                          dtc_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Schedule autotuner. Replaces the reference's hand-written schedule table   */
/* (scripts/DTCSpMM/run_DTC_SpMM.py:10-30: balance yes/no, vector width and   */
/* N split chosen per dataset and N) by measurement on the caller's data.     */
/* ------------------------------------------------------------------------- */
typedef struct {
  int32_t mode;   /* 0 = window-scheduled (no window split), 1 = strict balance */
  int32_t waves;  /* chunks = waves x SMs, capped at T: the split threshold is  */
                  /* ceil(T / chunks) TC blocks (one CTA per SM pulls chunks)  */
  int32_t ntile;  /* 128-feature tiles per CTA (1, 2 or 4)                      */
  int32_t grid;   /* chunk count the measurement used (output)                  */
  float ms;       /* mean kernel time over the timed repetitions (output)       */
} dtc_schedule;

/* Fills out[0..min(count, max_out)) with every schedule the kernels support for
 * N and returns the count (out may be NULL to query it): waves 1, 2, 4, 8, 16,
 * 32 and 64 in window mode, 1 to 16 in balance mode (whose cut windows keep
 * partial tiles per chunk), times the N-tiles the kernels hold for N. */
int dtc_schedule_candidates(int32_t N, dtc_schedule* out, int max_out);
/* The same for a given window height and kernel family (split = 1 for the
 * split-precision forms, whose N-tiles per CTA are capped at 2 at height 32). */
int dtc_schedule_candidates_ex(int32_t N, int32_t block_h, int split, dtc_schedule* out,
                               int max_out);

/* Workspace that every candidate's balance mode fits in. */
dtc_status dtc_autotune_workspace_bytes(int32_t num_nodes, int64_t num_blocks, int32_t N,
                                        int32_t block_h, size_t* bytes);

/* Times every candidate (one untimed run + `reps` runs between CUDA events on
 * `stream`; synchronises it; split forms at block width 16 skip N-tile counts
 * above 2, which those kernels cap) on the given ME-TCF arrays and B form, writes the
 * measured schedules to results[0..max_results), their count to *num_results
 * and the index of the fastest to *best. d_C receives the last candidate's
 * product. Arguments as in dtc_spmm_ex. */
dtc_status dtc_autotune(const int32_t* d_rowWindowOffset, const uint8_t* d_tileId,
                        const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                        const float* d_tcValues, int32_t num_nodes, int32_t num_windows,
                        int64_t num_blocks, int32_t block_h, int32_t block_w, int bformat,
                        const void* d_Bplane0,
                        const void* d_Bplane1, int32_t N, int precision, float* d_C,
                        void* d_workspace, size_t workspace_bytes, int reps,
                        dtc_schedule* results, int max_results, int* num_results, int* best,
                        dtc_stream_t stream);

/* ------------------------------------------------------------------------- */
/* Learned schedule cost model (no reference counterpart: the reference's     */
/* schedule is the fixed table of scripts/DTCSpMM/run_DTC_SpMM.py:10-30).      */
/* ------------------------------------------------------------------------- */

/* 48 structural features of a square CSR matrix and its ME-TCF form (row-length
 * histogram, TC blocks per window, nonzeros per block, column locality, sizes;
 * the layout is listed in the library's features source) into d_features[48].
 * Needs the ME-TCF row-window offsets, block offsets and edgeToColumn (the
 * conversion's in-place output). Bitwise reproducible. */
size_t dtc_features_workspace_bytes(void);
dtc_status dtc_features(const int32_t* d_rowptr, const int32_t* d_col, int32_t num_nodes,
                        int64_t nnz, const int32_t* d_rowWindowOffset,
                        const int32_t* d_tcblockOffset, const int32_t* d_edgeToColumn,
                        int32_t num_windows, int64_t num_blocks, int32_t N, float* d_features,
                        void* d_workspace, size_t workspace_bytes, dtc_stream_t stream);

/* MLP in -> h1 -> h2 -> out, ReLU hidden layers, linear output. Parameters are
 * one fp32 vector: W1[h1][in], b1[h1], W2[h2][h1], b2[h2], W3[out][h2], b3[out];
 * activations are row-major [batch][width]. */
typedef struct {
  int32_t in, h1, h2, out;
} dtc_mlp_dims;

/* Number of parameters, or -1 for invalid dims (each in [1, 4096]). */
int64_t dtc_mlp_num_params(const dtc_mlp_dims* dims);

/* Forward pass: d_H1[batch][h1], d_H2[batch][h2] (post-ReLU), d_Y[batch][out]. */
dtc_status dtc_mlp_forward(const dtc_mlp_dims* dims, const float* d_params, const float* d_X,
                           int32_t batch, float* d_H1, float* d_H2, float* d_Y,
                           dtc_stream_t stream);

/* Masked MSE loss L = sum mask*(Y-target)^2 / sum mask into *d_loss and its
 * gradient with respect to every parameter into d_grads (same layout as the
 * parameters), from the activations of dtc_mlp_forward. Deterministic. */
size_t dtc_mlp_backward_workspace_bytes(const dtc_mlp_dims* dims, int32_t batch);
dtc_status dtc_mlp_backward(const dtc_mlp_dims* dims, const float* d_params, const float* d_X,
                            const float* d_H1, const float* d_H2, const float* d_Y,
                            const float* d_target, const float* d_mask, int32_t batch,
                            float* d_grads, float* d_loss, void* d_workspace,
                            size_t workspace_bytes, dtc_stream_t stream);

/* One Adam step (bias-corrected, step >= 1) over n parameters. */
dtc_status dtc_mlp_adam(float* d_params, const float* d_grads, float* d_m, float* d_v, int64_t n,
                        float lr, float beta1, float beta2, float eps, int32_t step,
                        dtc_stream_t stream);

/* d_choice[r] = argmin over feasible outputs of d_Y[r][.] (lowest index on
 * ties, -1 if none is feasible). d_feasible: NULL (all), one row shared by all
 * (feasible_per_row = 0) or one row per input (feasible_per_row = 1). */
dtc_status dtc_mlp_argmin(const float* d_Y, const uint8_t* d_feasible, int feasible_per_row,
                          int32_t batch, int32_t out, int32_t* d_choice, dtc_stream_t stream);

/* Per-CTA timing of the SpMM kernels, for load-balance analysis; off by
 * default. While set on the current device (capacity > 0), every SpMM launch
 * writes, for each of its CTAs c < capacity (c = blockIdx.x + gridDim.x *
 * blockIdx.y), four uint64 values to d_records[4c .. 4c+3]: the %globaltimer
 * (ns) at kernel entry and at exit, the SM id, and the number of TC-block
 * chunks the CTA processed. capacity = 0 turns it off. No reference
 * counterpart (the reference's per-SM clock kernels,
 * DTC-SpMM/DTCSpMM_kernel.cu:62-79, are a separate instrumented build). */
dtc_status dtc_set_cta_timer(uint64_t* d_records, int32_t capacity);

/* d_rowWindowOffset[num_windows+1] from a sorted d_tcblockRowid[T]. */
dtc_status dtc_rowid_to_window_offset(const int32_t* d_tcblockRowid, int64_t num_blocks,
                                      int32_t num_windows, int32_t* d_rowWindowOffset,
                                      dtc_stream_t stream);

/* Legacy-ISA comparison kernel: the same product with sm_80-style
 * mma.sync.m16n8k8 TF32, one warp group per row window (the instruction
 * family of DTCSpMM_kernel.cu:2663-2866). Any N >= 1. */
dtc_status dtc_spmm_mma_sync(const int32_t* d_rowWindowOffset, const uint8_t* d_tileId,
                             const int32_t* d_tcblockOffset, const int32_t* d_sparseAToX,
                             const float* d_tcValues, int32_t num_nodes, int32_t num_windows,
                             const float* d_B, int32_t N, float* d_C, dtc_stream_t stream);

#ifdef __cplusplus
}  /* extern "C" */
#endif
#endif  /* DTC_SPMM_H_ */
