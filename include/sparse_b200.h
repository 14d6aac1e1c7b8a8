/*
 * sparse_b200.h -- C ABI of libsparse_b200.so, the B200 (sm_100a) sparse
 * hot path of SciWasm.Sparse.
 *
 * The reference's JavaScript module (src/sequential/src/sparse32.js and its
 * f64 twin sparse64.js) keeps every matrix as typed arrays in one wasm linear
 * memory and calls wasm exports with i32 byte offsets plus sizes, e.g.
 * `spmv_csr(rowptr, col, val, x, y, N)`
 * (src/sequential/src/sparse_opt_32.wat:227).  This ABI keeps that shape:
 * every array argument is a DEVICE pointer (allocate it with sb_malloc or any
 * CUDA allocator of the same process), every size is an integer, and each
 * call is ordered on the CUDA stream passed as `stream` (NULL = the legacy
 * default stream).  The f32 and f64 wasm modules become one entry point with
 * a dtype argument.  No torch type appears anywhere in this ABI.
 *
 * Status codes: every function returns SB_OK (0) or a negative SB_E* code;
 * sb_last_error() returns a message for the calling host thread.  Calls never
 * fall back to the CPU: without a usable CUDA device they return SB_ENODEV.
 *
 * Each declaration cites the reference interface it replaces (file:line,
 * relative to the SciWasm.Sparse project root).
 */
#ifndef SPARSE_B200_H
#define SPARSE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SB_OK 0
#define SB_EINVAL (-1)    /* bad argument (null pointer, negative size, bad dtype) */
#define SB_ENOMEM (-2)    /* device allocation failed */
#define SB_EREFUSED (-3)  /* conversion refused by the reference's admission test */
#define SB_ETIMEOUT (-4)  /* a bounded device wait ran out (dependency never ready) */
#define SB_ECUDA (-5)     /* CUDA runtime error (message in sb_last_error) */
#define SB_ENODEV (-6)    /* no CUDA device usable by this library */
#define SB_EALIGN (-7)    /* pointer misaligned for the requested path */

/* Value types.  SB_F32 / SB_F64 are the reference's *32 / *64 modules;
 * SB_BF16 is a storage-only type for SpMV values (FP32 accumulation). */
#define SB_F32 0
#define SB_F64 1
#define SB_BF16 2

/* ---------------------------------------------------------------------- */
/* Runtime: the stand-in for MatMachJS's _malloc/_free on wasm memory     */
/* (src/sequential/libs/matmachjs.wat:46-48) and for typed-array views.    */
/* ---------------------------------------------------------------------- */
int sb_version(void);
const char* sb_last_error(void);
const char* sb_status_string(int status);
int sb_device_count(int* count);
int sb_set_device(int device);
int sb_malloc(void** ptr, size_t bytes);
int sb_free(void* ptr);
int sb_host_alloc(void** ptr, size_t bytes); /* pinned host memory */
int sb_host_free(void* ptr);
int sb_memcpy_htod(void* dst, const void* src, size_t bytes, void* stream);
int sb_memcpy_dtoh(void* dst, const void* src, size_t bytes, void* stream);
int sb_memcpy_dtod(void* dst, const void* src, size_t bytes, void* stream);
int sb_memset(void* dst, int value, size_t bytes, void* stream);
int sb_stream_create(void** stream);
int sb_stream_destroy(void* stream);
/* A non-blocking stream with a scheduling priority (CUDA convention: a
 * numerically lower value is more urgent; clamped into the device's range,
 * which sb_stream_priority_range returns). */
int sb_stream_create_priority(void** stream, int priority);
int sb_stream_priority_range(int* least, int* greatest);
int sb_stream_synchronize(void* stream);
int sb_mem_info(size_t* free_bytes, size_t* total_bytes);
/* CUDA events for stream-ordered completion tracking and timing
 * (sb_event_query returns 1 when complete, 0 when not yet, < 0 on error). */
int sb_event_create(void** event);
int sb_event_destroy(void* event);
int sb_event_record(void* event, void* stream);
int sb_event_query(void* event);
int sb_event_synchronize(void* event);
int sb_event_elapsed_ms(void* start, void* end, float* ms);
/* Later work on `stream` waits for the event's recorded work. */
int sb_stream_wait_event(void* stream, void* event);
/* Synchronises the device, returns and clears its status word: 0, or the code
 * of a kernel whose bounded wait gave up (1 = bulk copy, 2 = dependency). */
int sb_device_status(int* code);

/* ---------------------------------------------------------------------- */
/* SpMV: y <- y + A x, repeated inner_max times (the *_wrapper exports).   */
/* ---------------------------------------------------------------------- */

/* Replaces spmv_coo / spmv_coo_wrapper
 * (src/sequential/src/sparse_opt_32.wat:175-225; dispatch
 * src/sequential/src/sparse32.js:1256-1262).  Any entry order is accepted. */
int sb_spmv_coo(int dtype, const int32_t* row, const int32_t* col, const void* val,
                const void* x, void* y, int32_t N, int64_t nnz, int32_t inner_max,
                void* stream);

/* sb_spmv_coo with flags; no counterpart in the reference.  SB_COO_ROWS_SORTED
 * states that row[] is non-decreasing (as in the reference's COO objects,
 * which create_COO_from_MM leaves sorted by (row, col)): rows that lie wholly
 * inside one 256-entry tile are then added without atomics (taken when the
 * mean row length is at most 16; longer rows keep the atomics, which cost
 * less there).  The flag is the caller's guarantee and is not checked: with
 * unsorted rows the result is wrong.  flags = 0 is sb_spmv_coo. */
#define SB_COO_ROWS_SORTED 1
int sb_spmv_coo_ex(int dtype, const int32_t* row, const int32_t* col, const void* val,
                   const void* x, void* y, int32_t N, int64_t nnz, int32_t inner_max,
                   int32_t flags, void* stream);

/* Replaces spmv_csr / spmv_csr_wrapper
 * (src/sequential/src/sparse_opt_32.wat:227-288; dispatch
 * src/sequential/src/sparse32.js:1264-1270).  nnz = row_ptr[N] is passed
 * explicitly so that no device read is needed to plan the launch.  Rows
 * without entries leave y untouched, as in the reference. */
int sb_spmv_csr(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                const void* x, void* y, int32_t N, int64_t nnz, int32_t inner_max,
                void* stream);

/* Kernel choice for CSR SpMV (no counterpart in the reference, whose
 * parallel harness picks among unrolled CSR variants per run,
 * src/parallel/tests/main32.js:150-313).  kernel 0 = row blocks (default),
 * 1 = streamed nonzero tiles (1024 per tile, 2048 with unroll = 2048; F32
 * and F64 with 16-byte aligned col/val, else row blocks), 2 = nonzero tiles
 * over row-aligned warp ranges (unroll = 256-nonzero tiles per warp, 1..64;
 * F32, F64 and BF16), 3 = block stream (a warp per 32-row block walks the
 * block's nonzeros in 256-entry chunks with vector loads; F32, F64 and BF16;
 * every row written once, no atomics); lanes_per_row 1..32 (power of two)
 * and unroll 2/4/8 tune the row-block kernel, 0 = chosen from the mean row
 * length; grid 0 = a resident grid striding over 32-row blocks (regular
 * rows), 1 = one warp per 32-row block (skewed row lengths). */
typedef struct sb_csr_opts {
  int32_t kernel;
  int32_t lanes_per_row;
  int32_t unroll;
  int32_t grid;
} sb_csr_opts;

/* sb_spmv_csr with explicit kernel options (opts may be NULL). */
int sb_spmv_csr_ex(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                   const void* x, void* y, int32_t N, int64_t nnz, int32_t inner_max,
                   const sb_csr_opts* opts, void* stream);

/* Row-sharded CSR SpMV with its all-gather fused into the stores (no
 * counterpart in the reference; the parallel reference shares one y in a
 * worker pool's memory).  The caller's rank holds rows [row_offset,
 * row_offset + rows) of the global matrix as a CSR of `rows` rows whose
 * columns keep their global numbers (x holds all columns).  For each of
 * those rows t = y_in[i] + sum_j A_ij x_j is computed by the row-block kernel
 * with `opts` (kernel 0; lanes, unroll, grid as in sb_spmv_csr_ex, so the
 * bits equal sb_spmv_csr_ex's with the same options) and stored to
 * dst[d][row_offset + i] for every d < ndst (1..8); rows without entries
 * store y_in[i] unchanged.  dst is a DEVICE array (8-byte aligned) of ndst
 * device pointers of full-length y buffers: this GPU's own, or other GPUs'
 * buffers mapped for peer access (stores over NVLink; no multicast); a
 * caller keeps it for the life of its exchange.  When every rank has run
 * its block into every rank's buffer and the ranks have synchronised, each
 * buffer holds the whole y.  dtype SB_F32, SB_F64, or SB_BF16 (bf16 values,
 * f32 vectors). */
int sb_spmv_csr_allgather(int dtype, const int32_t* row_ptr, const int32_t* col,
                          const void* val, const void* x, const void* y_in, int32_t rows,
                          int64_t nnz, int64_t row_offset, void* const* dst, int32_t ndst,
                          const sb_csr_opts* opts, void* stream);

/* Times the candidate kernel options around this matrix's row-length
 * statistics (reps calls each, on a scratch y) and returns the fastest in
 * *best (and its time per call in *best_ms).  Returns after timing. */
int sb_csr_autotune(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                    const void* x, int32_t N, int64_t nnz, int32_t reps, sb_csr_opts* best,
                    float* best_ms, void* stream);

/* Format and kernel choice for SpMV on one CSR matrix (no counterpart in the
 * reference, whose users pick coo_csr / csr_dia / csr_ell by hand,
 * src/sequential/src/sparse32.js:1436-1720).  From the matrix's statistics
 * (N, nnz, max row length nc, diagonal count nd) it records which of DIA and
 * ELL the reference's admission test allows and the compulsory bytes of one
 * y <- y + A x per format (bytes[]: CSR, DIA, ELL, COO).
 *   mode SB_TUNE_MODEL: format = the admitted format with the fewest bytes,
 *     csr = options from the row-length statistics; nothing is timed (x may
 *     be NULL).
 *   mode SB_TUNE_TIMED: every admitted format within twice the CSR bytes is
 *     timed on the device (reps calls each on a scratch y; ms[] per format,
 *     -1 when not timed): CSR with the options of sb_csr_autotune, DIA and
 *     ELL built into scratch, COO with rows expanded from row_ptr; format =
 *     the fastest, csr = the best CSR options.  BF16 values time CSR only.
 * format is SB_FMT_CSR, SB_FMT_DIA, SB_FMT_ELL or SB_FMT_COO.  Returns when
 * done; the matrix itself is not changed. */
#define SB_TUNE_MODEL 0
#define SB_TUNE_TIMED 1
#define SB_FMT_CSR 0
#define SB_FMT_DIA 1
#define SB_FMT_ELL 2
#define SB_FMT_COO 3
typedef struct sb_spmv_choice {
  int32_t format;
  sb_csr_opts csr;
  int32_t ndiags;
  int32_t ncols;
  int32_t dia_admitted;
  int32_t ell_admitted;
  float ms[4];
  int64_t bytes[4];
} sb_spmv_choice;
int sb_spmv_autotune(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                     const void* x, int32_t N, int64_t nnz, int32_t mode, int32_t reps,
                     sb_spmv_choice* choice, void* stream);

/* The COO form of a CSR matrix (no counterpart in the reference): coo_row
 * expanded from row_ptr (rows non-decreasing, so SB_COO_ROWS_SORTED holds),
 * col and val copied; outputs caller-allocated, stream-ordered. */
int sb_csr_coo(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val, int32_t N,
               int64_t nnz, int32_t* coo_row, int32_t* coo_col, void* coo_val, void* stream);

/* The floor of an SpMV on this matrix (no counterpart in the reference):
 * *out += sum over k of val[k] * x[col[k]] (the sum of all entries of A x),
 * accumulated per warp in the value type and added to *out (a device double)
 * with one atomic per warp.  It reads the column and value streams an SpMV
 * must read and gathers x once per entry, with no row structure, so its time
 * bounds every SpMV kernel on the same col/val/x from below.  col and val
 * must be 16-byte aligned. */
int sb_gather_dot(int dtype, const int32_t* col, const void* val, const void* x, int64_t nnz,
                  double* out, void* stream);

/* The gather floor of several right-hand sides (no counterpart in the
 * reference): *out = sum over k of val[k] * (sum over h < nrhs of
 * x[col[k]*nrhs + h]), x holding x_rows rows of nrhs values (row-major, as
 * sb_batch_item's x).  It streams col and val and gathers each entry's x row
 * with the loads the batched SpMV uses, nothing else: the floor of a batched
 * SpMV over the same entries.  dtype SB_F32, SB_F64, or SB_BF16 (bf16 values,
 * f32 x).  out is a device double. */
int sb_gather_dot_rows(int dtype, const int32_t* col, const void* val, const void* x,
                       int64_t x_rows, int32_t nrhs, int64_t nnz, double* out, void* stream);

/* Reduced-precision storage (no counterpart in the reference, which keeps
 * f32 or f64 values): sb_spmv_csr / sb_spmv_csr_ex accept dtype SB_BF16 for
 * BF16-stored values with f32 x, y and f32 accumulation (long rows use
 * compensated sums).  sb_convert_values converts a value array between
 * SB_F32, SB_F64 and SB_BF16 (round to nearest even). */
int sb_convert_values(int src_dtype, const void* src, int dst_dtype, void* dst, int64_t n,
                      void* stream);

/* Replaces spmv_dia / spmv_dia_wrapper
 * (src/sequential/src/sparse_opt_32.wat:290-425; dispatch
 * src/sequential/src/sparse32.js:1272-1278).  offset[nd] diagonal offsets
 * (device), data[nd*stride] diagonal-major.  dtype SB_BF16 (no counterpart in
 * the reference): BF16 data with f32 x, y and sums in the same per-row
 * order. */
int sb_spmv_dia(int dtype, const int32_t* offset, const void* data, int32_t N, int32_t nd,
                int32_t stride, const void* x, void* y, int32_t inner_max, void* stream);

/* Replaces spmv_ell / spmv_ell_wrapper
 * (src/sequential/src/sparse_opt_32.wat:427-498; dispatch
 * src/sequential/src/sparse32.js:1280-1286).  Column-major indices/data of
 * nc*N slots; padding slots (data 0, index 0) are applied like the reference. */
int sb_spmv_ell(int dtype, const int32_t* indices, const void* data, int32_t N, int32_t nc,
                const void* x, void* y, int32_t inner_max, void* stream);

/* ---------------------------------------------------------------------- */
/* Batched SpMV (no counterpart in the reference, which calls spmv once per  */
/* matrix and vector, src/sequential/src/sparse32.js:1232-1286).            */
/* ---------------------------------------------------------------------- */

/* One matrix of a batch: y <- y + A x for nrhs (1..8) right-hand sides, x
 * and y stored N x nrhs row-major (x[col*nrhs + j]).  flags bit 0 set:
 * y <- A x (y is overwritten, rows without entries get 0).  Other flag bits
 * must be 0.  The y ranges of
 * different items must not overlap (x may be shared).
 *   format SB_FMT_CSR (0): row_ptr[N+1], col[nnz], val[nnz]; lanes: lanes
 *     per row (1..32, power of two), 0 = chosen from nnz/N (from nnz/(2N)
 *     with nrhs >= 2).  With nrhs >= 2
 *     and x 16-byte aligned, lanes 1 = one row per lane with the nrhs sums in
 *     registers, lanes >= 2 = that many lanes interleaved over a row, each
 *     with nrhs partial sums (x rows loaded as vectors in both); with x not
 *     16-byte aligned the nrhs right-hand sides go across lanes.
 *   format SB_FMT_DIA (1): row_ptr = offsets[width] (ascending, as csr_dia
 *     makes them), val = data[width*N] diagonal-major (stride N); each row is
 *     bit-identical to sb_spmv_dia (the reference's per-row order).
 *   format SB_FMT_ELL (2): col = indices[width*N] and val = data[width*N],
 *     column-major; each row is bit-identical to sb_spmv_ell.
 * Zero-initialised trailing fields (format 0, width 0) describe a CSR item. */
typedef struct sb_batch_item {
  const int32_t* row_ptr;
  const int32_t* col;
  const void* val;
  const void* x;
  void* y;
  int32_t N;
  int32_t nrhs;
  int32_t lanes;
  int32_t flags;
  int64_t nnz;
  int32_t format;
  int32_t width;
} sb_batch_item;

typedef struct sb_batch_exec sb_batch_exec;

/* An executor for batches of up to `capacity` matrices whose values are
 * stored as dtype (SB_F32, SB_F64 or SB_BF16 with f32 vectors).  It holds two
 * descriptor sets, each with a captured CUDA graph: descriptor upload,
 * work-counter reset and the persistent kernel over all 32-row blocks of the
 * batch.  Runs alternate between the sets. */
int sb_batch_exec_create(int dtype, int32_t capacity, sb_batch_exec** exec);
int sb_batch_exec_destroy(sb_batch_exec* exec);
/* Launch the graph for items[0..n) on `stream` (stream-ordered).  The call
 * waits only for the run before the previous one (the last user of this
 * run's descriptor set), so a run can be staged while the previous one
 * executes. */
int sb_batch_exec_run(sb_batch_exec* exec, const sb_batch_item* items, int32_t n, void* stream);

/* ---------------------------------------------------------------------- */
/* Format conversions (bit-exact with the reference).  These calls return */
/* after the device work is complete (they may read results to the host). */
/* CSR inputs must have monotone row_ptr with row_ptr[0] = 0 and columns  */
/* in [0, N); COO indices are checked on the device (SB_EINVAL).          */
/* ---------------------------------------------------------------------- */

/* Replaces coo_csr (src/sequential/src/sparse32.js:1674-1720 with the
 * per-row stable sort :1612-1627; FP64 src/sequential/src/sparse64.js:1255).
 * Outputs: csr_row_ptr[N+1], csr_col[nnz], csr_val[nnz] (caller-allocated,
 * as allocate_CSR :2252 does); entries are stably ordered by (row, col). */
int sb_coo_csr(int dtype, const int32_t* row, const int32_t* col, const void* val, int32_t N,
               int64_t nnz, int32_t* csr_row_ptr, int32_t* csr_col, void* csr_val, void* stream);

/* Replaces coo_csc (src/sequential/src/sparse32.js:1629-1671): the CSC
 * (col_ptr[N+1], row[nnz], val[nnz]) with entries stably ordered by
 * (col, row), as the reference's count / scatter / per-column stable sort. */
int sb_coo_csc(int dtype, const int32_t* row, const int32_t* col, const void* val, int32_t N,
               int64_t nnz, int32_t* csc_col_ptr, int32_t* csc_row, void* csc_val,
               void* stream);

/* Replaces num_cols (src/sequential/src/sparse32.js:1436-1447): the maximum
 * row length, returned to the host in *nc. */
int sb_num_cols(const int32_t* row_ptr, int32_t N, int32_t* nc, void* stream);

/* The admission test of csr_ell (src/sequential/src/sparse32.js:1457):
 * returns 1 when nc*N < 2^27 and nc*N/nnz <= 5 (in doubles), else 0. */
int sb_ell_admitted(int64_t ncols, int32_t N, int64_t nnz);

/* Replaces the fill of csr_ell (src/sequential/src/sparse32.js:1449-1484).
 * Returns SB_EREFUSED (writing nothing) where the reference returns
 * undefined.  indices/data hold nc*N column-major slots, zero padded. */
int sb_csr_ell(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val, int32_t N,
               int64_t nnz, int32_t nc, int32_t* indices, void* data, void* stream);

/* Replaces num_diags (src/sequential/src/sparse32.js:1486-1512): number of
 * occupied diagonals in *nd, *stride = N. */
int sb_num_diags(const int32_t* row_ptr, const int32_t* col, int32_t N, int32_t* nd,
                 int32_t* stride, void* stream);

/* The admission test of csr_dia (src/sequential/src/sparse32.js:1525). */
int sb_dia_admitted(int64_t ndiags, int32_t stride, int64_t nnz);

/* Replaces the fill of csr_dia (src/sequential/src/sparse32.js:1515-1574):
 * offset[nd] ascending, data[nd*stride] diagonal-major (zero where no entry),
 * a later duplicate (i, c) in row order overwriting an earlier one.  Returns
 * SB_EREFUSED where the reference returns undefined. */
int sb_csr_dia(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val, int32_t N,
               int64_t nnz, int32_t nd, int32_t stride, int32_t* offset, void* data,
               void* stream);

/* ---------------------------------------------------------------------- */
/* Level sets and sparse triangular solves                                */
/* ---------------------------------------------------------------------- */
typedef struct sb_spts_plan sb_spts_plan;

#define SB_SPTS_LEVEL 0    /* level by level (row kernel arithmetic)        */
#define SB_SPTS_SYNCFREE 1 /* natural order, ready flags (sync-free order)  */
#define SB_SPTS_HYBRID 2   /* level order, ready flags (row kernel order)   */

#define SB_SPTS_ACC_NATIVE 0 /* accumulate and divide in the value type      */
#define SB_SPTS_ACC_F64 1    /* f32 values: accumulate and divide in f64     */

/* Replaces CSR_create_level_sets / CSR_create_level_sets_with_reorder
 * (src/parallel/src/sparse32.js:2942-3181; older copy
 * src/parallel/src/spts32.js:158-357).  Computes, bit-exactly, the level of
 * every row, level_ptr, the stable permutation by level, its inverse
 * (`order`) and the level-reordered CSR with relabelled columns.  The
 * caller's row_ptr/col/val must outlive the plan (the sync-free solve reads
 * them).  Returns after the analysis is complete. */
int sb_spts_analyze(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                    int32_t N, int64_t nnz, void* stream, sb_spts_plan** plan);
int sb_spts_plan_destroy(sb_spts_plan* plan);
/* nlevels; solvable = 1 when every row ends with its diagonal and all other
 * columns are below it (the solves' precondition). */
int sb_spts_plan_info(const sb_spts_plan* plan, int32_t* nlevels, int32_t* solvable);
/* Device time of the analysis (no counterpart in the reference): milliseconds
 * between CUDA events recorded on the analysis stream before its first
 * kernel and after its last, after the plan's one allocation. */
int sb_spts_plan_analysis_ms(const sb_spts_plan* plan, float* ms);
/* Device-to-device copies of the analysis results (any pointer may be NULL):
 * level[N], level_ptr[nlevels+1], permutation[N], order[N]. */
int sb_spts_plan_levels(const sb_spts_plan* plan, int32_t* level, int32_t* level_ptr,
                        int32_t* permutation, int32_t* order, void* stream);
/* The level-reordered CSR (row_ptr[N+1], col[nnz], val[nnz]). */
int sb_spts_plan_reordered(const sb_spts_plan* plan, int32_t* row_ptr, int32_t* col, void* val,
                           void* stream);

/* Solve L y = b (b, y in natural row order).  SB_SPTS_LEVEL replaces
 * spts_level_csr (src/parallel/src/sparse_opt_32.wat:11759;
 * src/parallel/src/spts_opt_32.wat:339-546), SB_SPTS_SYNCFREE replaces
 * spts_csr_sync_free (src/parallel/src/spts_opt_32.wat:8-260) and
 * SB_SPTS_HYBRID replaces spts_csr_opt_level_sync_free
 * (src/parallel/src/sparse_opt_32.wat:12846-13445).  Stream-ordered; a
 * dependency wait that runs out is reported by sb_device_status (code 2). */
int sb_spts_solve(const sb_spts_plan* plan, int algo, int policy, const void* b, void* y,
                  void* stream);

/* Replaces spts_csc / spts_csc_wrapper (src/sequential/src/sparse_opt_32.wat:11-148;
 * test driver src/sequential/src/sparse32.js:1845-1870): y = x, then for
 * each column j, y_j /= L_jj (the column's first entry) and y_r -= L_rj*y_j
 * for the rest of the column.  Every row thus subtracts in increasing column
 * order before its division, the sync-free kernel's arithmetic on L in CSR,
 * which is what runs here (after a device transpose); results are
 * bit-identical to the reference's column sweep.  The matrix must be a CSC
 * lower triangle with each column starting at its diagonal (SB_EINVAL
 * otherwise).  Returns after the solve. */
int sb_spts_csc(int dtype, const int32_t* col_ptr, const int32_t* row, const void* val,
                int32_t N, int64_t nnz, const void* x, void* y, void* stream);

/* Replaces the raw spts_csr_sync_free export on caller arrays without any
 * structural check: every dependency wait is bounded by spin_limit_cycles
 * (SM clock cycles, <= 0 for the default of about a second) and a wait that
 * runs out makes the call return SB_ETIMEOUT instead of hanging.  Returns
 * after the solve. */
int sb_spts_syncfree_csr(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                         int32_t N, const void* b, void* y, int64_t spin_limit_cycles,
                         void* stream);

/* No counterpart in the reference (its wasm memory is allocated by the JS
 * host; this is an addition for callers that cannot allocate device memory).
 * Same solve as sb_spts_syncfree_csr, but the ready flags, row ticket and
 * status word live in a fixed 16 MiB device array inside the library, so the
 * call makes no device allocation: for callers whose device memory is all
 * reserved up front (a serving process that admitted its matrices against a
 * fixed HBM budget, an embedding runtime that owns every device allocation)
 * or that must not pay cudaMalloc's synchronisation in a latency-critical
 * loop.  Limit: N <= 4,194,304 rows (larger N returns SB_EINVAL).  The first
 * call on a device looks up the array's device address (do that call before
 * any stream capture).  Every call on a device shares the array: calls that
 * overlap on the GPU (other streams, other host threads) race and must be
 * serialised by the caller.  Returns after the solve. */
int sb_spts_syncfree_csr_noalloc(int dtype, const int32_t* row_ptr, const int32_t* col,
                                 const void* val, int32_t N, const void* b, void* y,
                                 int64_t spin_limit_cycles, void* stream);

/* Growth estimate of a triangular factor (no counterpart in the reference):
 * max over rows of sum_{j<i} |L_ij| / |L_ii| (inf for a zero diagonal).  Below
 * 1 the factor is row diagonally dominant and a solve in the value type does
 * not amplify rounding; above a threshold the caller flags the factor for
 * SB_SPTS_ACC_F64.  Returns after the reduction. */
int sb_spts_plan_growth(const sb_spts_plan* plan, double* growth, void* stream);

/* Batched solves (no counterpart in the reference, which solves one system
 * per call): many independent systems, each with its own analysed plan, in
 * one persistent launch replayed from a captured CUDA graph.  Every row is
 * solved with the arithmetic of SB_SPTS_HYBRID, so each result is
 * bit-identical to sb_spts_solve(plan, SB_SPTS_HYBRID, policy, b, y).  An
 * executor serves one value dtype (SB_F32 or SB_F64) and one accumulation
 * policy.  A solve keeps its rows' values, published with a pending
 * sentinel, in a work vector of N values of the plan's dtype: the plan's own
 * (work = NULL), or one the caller gives (work != NULL, aligned to the value
 * size, not shared with any solve in flight; no counterpart in the
 * reference).  Solves on the plan's own vector must be ordered (one stream,
 * or events) and a plan may appear once per run with it; solves with their
 * own work vectors may repeat a plan in one run and run concurrently with
 * other runs on the same plan.  Stream-ordered; a dependency wait that runs
 * out is reported by sb_device_status (code 2). */
typedef struct sb_spts_batch sb_spts_batch;
typedef struct sb_spts_batch_item {
  sb_spts_plan* plan;
  const void* b; /* right-hand side, natural row order */
  void* y;       /* solution, natural row order        */
  void* work;    /* N values of the plan's dtype, or NULL (the plan's own) */
} sb_spts_batch_item;
int sb_spts_batch_create(int dtype, int policy, int32_t capacity, sb_spts_batch** out);
int sb_spts_batch_destroy(sb_spts_batch* e);
int sb_spts_batch_run(sb_spts_batch* e, const sb_spts_batch_item* items, int32_t n,
                      void* stream);
/* Launch shape of later runs: blocks_per_sm 0 (the default) launches one warp
 * per 32-row chunk, resident blocks capped by the batch size; > 0 launches at
 * most that many blocks per SM (and no more than fit), whose warps take
 * chunks until the batch is done, so that a run leaves SMs to work on other
 * streams (for instance a second executor's run). */
int sb_spts_batch_set_grid(sb_spts_batch* e, int32_t blocks_per_sm);

/* ---------------------------------------------------------------------- */
/* Reductions over a row-sorted COO (rows non-decreasing, as the           */
/* reference's quick-sorted objects are; unsorted rows return SB_EINVAL).  */
/* Each returns after a sortedness check that reads back one flag.         */
/* ---------------------------------------------------------------------- */

/* Replaces diagonal_coo (src/sequential/src/sparse_opt_32.wat:1707-1798;
 * JS A.diagonal(offset), src/sequential/src/sparse32.js:314-321): diag[i] =
 * the first entry of row start+i in column start+i+k (start = max(0, -k)),
 * else 0, for N - |k| slots.  |k| >= N returns SB_EINVAL (the reference
 * returns no vector). */
int sb_diagonal_coo(int dtype, int32_t k, const int32_t* row, const int32_t* col,
                    const void* val, void* diag, int32_t N, int64_t nnz, void* stream);
/* Replaces min_coo (src/sequential/src/sparse_opt_32.wat:1847-1946; JS
 * A.min(axis), src/sequential/src/sparse32.js:323-328): axis 1 gives each
 * row's minimum, 0 when the row has fewer than N entries and its minimum is
 * positive, with the reference's walk reproduced exactly (an empty row
 * repeats the previous stored minimum when that is <= 0; the last entry's
 * row stays 0 when it holds one entry; later rows stay 0).  Other axes leave
 * out unchanged (the caller zero-fills it, as create_vec does). */
int sb_min_coo(int dtype, int32_t axis, const int32_t* row, const int32_t* col, const void* val,
               void* out, int32_t N, int64_t nnz, void* stream);
/* sum_coo (src/sequential/src/sparse_opt_32.wat:1800-1845), axis 1: the sum
 * of each row in storage order.  The reference's export advances its row
 * counter for every entry it adds as well, so its output is not this row
 * sum (it is not reachable from the JS API). */
int sb_sum_coo(int dtype, int32_t axis, const int32_t* row, const int32_t* col, const void* val,
               void* out, int32_t N, int64_t nnz, void* stream);

/* ---------------------------------------------------------------------- */
/* Row reordering (src/parallel/src/sparse32.js:2148-2269).                */
/* ---------------------------------------------------------------------- */

/* Replaces sort_rows_by_nnz (:2148-2218): the rows stably sorted by their
 * number of nonzeros (ascending) into a new CSR (columns unchanged);
 * permutation[new] = old row, nnz_per_row = the new matrix's row lengths,
 * small_rows[q] (host, may be NULL) = rows with at most q nonzeros, q = 0..3
 * (num_zero_rows .. num_three_rows).  Returns after the device work. */
int sb_sort_rows_by_nnz(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                        int32_t N, int64_t nnz, int32_t* out_row_ptr, int32_t* out_col,
                        void* out_val, int32_t* nnz_per_row, int32_t* permutation,
                        int32_t* small_rows, void* stream);
/* Replaces sort_y_rows_by_nnz (:2220-2235): out[permutation[i]] = in[i]
 * (a result of the reordered matrix back in the original row order). */
int sb_unpermute_rows(int dtype, const int32_t* permutation, const void* in, void* out,
                      int32_t N, void* stream);
/* Replaces reorder_NN (src/parallel/src/sparse32.js:2501-2622, with
 * reorder_subset :2415-2483, find_next_row :2321-2394 and
 * assign_w_min_elems :2271-2318): a nearest-neighbour row order.  From the
 * first non-empty row on, consecutive position ranges sized by the
 * row-length histogram (at most 1024 rows; with rows sorted by length, as the
 * reference calls it on sort_rows_by_nnz's output, each range holds rows of
 * one length) are walked greedily: each visited row joins a window of the
 * last w (1..32) rows, each window row keeps the w unvisited rows of its
 * range with the highest Jaccard similarity of 16-column cache lines, and the
 * next row is the best first candidate over the window.  Bit-exact with the
 * reference: walk[N] (input row at each new position; positions no walk
 * reaches keep their index), perm_out[N] = perm_in[walk[i]] (perm_in NULL =
 * the identity), and the reordered CSR (rows gathered in walk order; the
 * reference's new row_ptr view is empty, so it writes no row pointers --
 * here they are written).  Returns after the device work. */
int sb_reorder_nn(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                  int32_t N, int64_t nnz, int32_t w, const int32_t* perm_in, int32_t* walk,
                  int32_t* perm_out, int32_t* out_row_ptr, int32_t* out_col, void* out_val,
                  void* stream);
/* Replaces calculate_csr_locality_index (:2238-2269): the percentage of
 * accesses whose 16-column line was last touched fewer than 16 rows before
 * (NaN for an empty matrix, as the reference's 0/0).  Returns after the
 * device work. */
int sb_csr_locality_index(const int32_t* row_ptr, const int32_t* col, int32_t N, int64_t nnz,
                          double* index, void* stream);

/* ---------------------------------------------------------------------- */
/* Matrix Market input: replaces mmread / read_matrix_MM_files /            */
/* create_COO_from_MM / create_LCOO_from_MM                                  */
/* (src/sequential/src/sparse32.js:1889-2172, 2499-2510).                    */
/* ---------------------------------------------------------------------- */
#define SB_MM_REAL 0
#define SB_MM_INTEGER 1
#define SB_MM_PATTERN 2
#define SB_MM_COMPLEX 3 /* the real part is read, as the reference's Number() of field 3 */

typedef struct sb_mm_header {
  int64_t nrows;
  int64_t ncols;
  int64_t nentries;    /* entry lines in the file */
  int32_t field;       /* SB_MM_* */
  int32_t symmetric;   /* 1 for the symmetry "symmetric"; anything else reads as general */
  int64_t data_offset; /* byte offset of the first line after the size line */
} sb_mm_header;

/* Host only (no device work): parses the banner ("%%MatrixMarket matrix
 * coordinate <field> <symmetry>", read_MM_header :1889-1911), skips comment
 * and blank lines and reads the size line.  Refuses more than 2^27 entries
 * (the reference throws, :1963-1965). */
int sb_mm_read_header(const char* text, size_t len, sb_mm_header* header);
/* Host only: parses the entry lines after the size line into host arrays
 * (1-based row/col as in the file, f64 values; val unused for pattern),
 * splitting the text across nthreads threads (<= 0: all hardware threads).
 * The number of entry lines must equal header->nentries. */
int sb_mm_read_entries(const char* text, size_t len, const sb_mm_header* header, int32_t* row,
                       int32_t* col, double* val, int32_t nthreads);
/* Device: the COO of create_COO_from_MM (lower = 0: explicit zeros dropped,
 * off-diagonal entries of symmetric files mirrored, :2103-2172) or of
 * create_LCOO_from_MM (lower = 1: the strictly lower part, upper entries of
 * symmetric files mirrored, then a unit diagonal, :1983-2099), sorted by
 * (row, col) in place of quick_sort_COO.  row/col/val are the device copies
 * of sb_mm_read_entries' arrays.  With out_row == NULL only *nnz is computed
 * (allocate, then call again).  Refuses more than 2^28 nonzeros.  Returns
 * after the device work is complete. */
int sb_mm_coo(int dtype, int lower, const sb_mm_header* header, const int32_t* row,
              const int32_t* col, const double* val, int32_t* out_row, int32_t* out_col,
              void* out_val, int64_t* nnz, void* stream);

/* ---------------------------------------------------------------------- */
/* eliminate_zeros and transpose (bit-exact with the reference's kernels). */
/* The nonzero test is v > 0 || v < 0 (+0, -0 and NaN count as zeros).    */
/* Calls that return a count return after the device work is complete.    */
/* ---------------------------------------------------------------------- */

/* Replaces count_nonzeros_coo (src/sequential/src/sparse_opt_32.wat:500),
 * used for COO and CSR values (src/sequential/src/sparse32.js:1140-1175). */
int sb_count_nonzeros(int dtype, const void* val, int64_t n, int64_t* count, void* stream);
/* Replaces copy_nonzeros_coo (src/sequential/src/sparse_opt_32.wat:523-546). */
int sb_copy_nonzeros_coo(int dtype, const int32_t* row, const int32_t* col, const void* val,
                         int64_t nnz, int32_t* orow, int32_t* ocol, void* oval, void* stream);
/* Replaces copy_nonzeros_csr (src/sequential/src/sparse_opt_32.wat:548-595)
 * over the N rows (out_row_ptr[N+1] rebuilt). */
int sb_copy_nonzeros_csr(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                         int32_t N, int64_t nnz, int32_t* orow_ptr, int32_t* ocol, void* oval,
                         void* stream);
/* Replaces count_nonzeros_dia (src/sequential/src/sparse_opt_32.wat:1948-2039). */
int sb_count_nonzeros_dia(int dtype, const int32_t* offset, const void* data, int32_t nd,
                          int32_t stride, int32_t N, int32_t* count_diags, int64_t* count,
                          void* stream);
/* Replaces copy_nonzeros_dia (src/sequential/src/sparse_opt_32.wat:2041-2134):
 * diagonals without nonzeros are dropped and each kept diagonal's nonzeros
 * are packed contiguously from its first in-band row, as the reference does;
 * odata (count_diags*stride) is zero-filled by the call. */
int sb_copy_nonzeros_dia(int dtype, const int32_t* offset, const void* data, int32_t nd,
                         int32_t stride, int32_t N, int32_t* ooffset, void* odata, void* stream);
/* Replaces count_nonzeros_ell (src/sequential/src/sparse_opt_32.wat:5821-5893). */
int sb_count_nonzeros_ell(int dtype, const void* data, int32_t nc, int32_t N, int32_t* count_cols,
                          int64_t* count, void* stream);
/* Replaces copy_nonzeros_ell (src/sequential/src/sparse_opt_32.wat:5895-5947):
 * each row's nonzeros packed in slot order into out_nc column-major slots. */
int sb_copy_nonzeros_ell(int dtype, const void* data, const int32_t* indices, int32_t nc,
                         int32_t N, int32_t out_nc, void* odata, int32_t* oindices, void* stream);
/* Replaces the COO branch of transpose (src/sequential/src/sparse32.js:1106-1115):
 * row and column arrays exchanged, no re-sort. */
int sb_transpose_coo(int dtype, const int32_t* row, const int32_t* col, const void* val,
                     int64_t nnz, int32_t* orow, int32_t* ocol, void* oval, void* stream);
/* Replaces transpose_csr (src/sequential/src/sparse_opt_32.wat:6348-6477). */
int sb_transpose_csr(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                     int32_t N, int64_t nnz, int32_t* orow_ptr, int32_t* ocol, void* oval,
                     void* stream);
/* Replaces transpose_dia (src/sequential/src/sparse_opt_32.wat:6479-6572):
 * offsets negated in their stored order; out-of-band slots are zeroed. */
int sb_transpose_dia(int dtype, const int32_t* offset, const void* data, int32_t nd,
                     int32_t stride, int32_t N, int32_t* ooffset, void* odata, void* stream);
/* Replaces count_transpose_cols_ell (src/sequential/src/sparse_opt_32.wat:6574-6632). */
int sb_count_transpose_cols_ell(int dtype, const void* data, const int32_t* indices, int32_t nc,
                                int32_t N, int32_t* count_cols, void* stream);
/* Replaces transpose_ell (src/sequential/src/sparse_opt_32.wat:6634-6701);
 * padding slots of the output are zeroed. */
int sb_transpose_ell(int dtype, const void* data, const int32_t* indices, int32_t nc, int32_t N,
                     int32_t out_nc, void* odata, int32_t* oindices, void* stream);

/* ---------------------------------------------------------------------- */
/* Element-wise maps                                                      */
/* ---------------------------------------------------------------------- */
#define SB_MAP_EXPM1 0
#define SB_MAP_LOG1P 1
#define SB_MAP_SIN 2
#define SB_MAP_TAN 3
#define SB_MAP_POW 4      /* p = exponent */
#define SB_MAP_DEG2RAD 5  /* p = pi (the reference passes Math.PI) */
#define SB_MAP_RAD2DEG 6  /* p = pi */
#define SB_MAP_SIGN 7
#define SB_MAP_ABS 8
#define SB_MAP_NEG 9
#define SB_MAP_SQRT 10
#define SB_MAP_CEIL 11
#define SB_MAP_FLOOR 12
#define SB_MAP_TRUNC 13
#define SB_MAP_NEAREST 14 /* round half to even */
#define SB_MAP_MULTIPLY 15 /* p = scalar */

/* Replaces the *_coo maps (src/sequential/src/sparse_opt_32.wat:597-1699),
 * applied to COO and CSR value arrays (src/sequential/src/sparse32.js:671-1104);
 * in == out is the in-place form. */
int sb_map_coo(int dtype, int op, double p, const void* in, void* out, int64_t n, void* stream);
/* Replaces the *_ell maps (src/sequential/src/sparse_opt_32.wat:4977-6346):
 * every one of the ncols*N slots, padding included. */
int sb_map_ell(int dtype, int op, double p, const void* in, void* out, int32_t ncols, int32_t N,
               void* stream);
/* Replaces the *_dia maps (src/sequential/src/sparse_opt_32.wat:2137-4976):
 * in-band slots only. */
int sb_map_dia(int dtype, int op, double p, const int32_t* offset, const void* in, void* out,
               int32_t ndiags, int32_t stride, int32_t N, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SPARSE_B200_H */
