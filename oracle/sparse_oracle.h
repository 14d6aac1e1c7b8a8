/*
 * sparse_oracle.h -- CPU restatement of SciWasm.Sparse's sparse kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the correctness oracle and the
 * timed CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / --impl reference leg may load it; the product path
 * (libsparse_b200.so and the sciwasm.sparse_b200 package) never does.
 *
 * Parity status: the functions that restate the reference's WebAssembly
 * kernels (SpMV in four formats, eliminate_zeros, transposes, diagonal/min
 * reductions, the exact element-wise maps, the CSC, sync-free and level-set
 * triangular solves) are PINNED bit for bit to outputs of those kernels,
 * executed from the reference's .wat text by tests/golden/wat_machine.py
 * (vectors in tests/golden/wat_vectors.npz, checked by
 * tests/test_wat_vectors.py).  The restatements of its JavaScript functions
 * (coo_csr, coo_csc, quick_sort_COO, csr_ell, csr_dia, static_nnz, the level
 * sets, Matrix Market input, row reorderings including reorder_NN) are PINNED
 * the same way to those functions executed from their source by
 * tests/golden/js_machine.py (tests/golden/js_vectors.npz,
 * tests/test_js_vectors.py).  Every function below restates one reference
 * function line by line (cited as file:line, paths relative to the
 * SciWasm.Sparse project root) and is compiled with -ffp-contract=off so that
 * wasm's separate mul/add (wasm has no FMA) is reproduced bit for bit.
 *
 * Index arrays are int32 as in the reference (i32 in wasm linear memory).
 * Counts that can exceed 2^31 in this build's workloads are int64.
 */
#ifndef SPARSE_ORACLE_H
#define SPARSE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- SpMV (y += A x), serial storage order ---------------- */
/* src/sequential/src/sparse_opt_32.wat:175-202 (spmv_coo), :227-271
 * (spmv_csr), :290-407 (spmv_dia), :427-479 (spmv_ell); the f64 module
 * src/sequential/src/sparse_opt_64.wat:187/239/302/439 is the same loop. */
void or_spmv_coo_f32(const int32_t* row, const int32_t* col, const float* val,
                     const float* x, float* y, int64_t nnz);
void or_spmv_coo_f64(const int32_t* row, const int32_t* col, const double* val,
                     const double* x, double* y, int64_t nnz);
void or_spmv_csr_f32(const int32_t* row_ptr, const int32_t* col, const float* val,
                     const float* x, float* y, int32_t N);
void or_spmv_csr_f64(const int32_t* row_ptr, const int32_t* col, const double* val,
                     const double* x, double* y, int32_t N);
void or_spmv_dia_f32(const int32_t* offset, const float* data, int32_t N, int32_t nd,
                     int32_t stride, const float* x, float* y);
void or_spmv_dia_f64(const int32_t* offset, const double* data, int32_t N, int32_t nd,
                     int32_t stride, const double* x, double* y);
void or_spmv_ell_f32(const int32_t* indices, const float* data, int32_t N, int32_t nc,
                     const float* x, float* y);
void or_spmv_ell_f64(const int32_t* indices, const double* data, int32_t N, int32_t nc,
                     const double* x, double* y);

/* Extended-precision "truth" y += A x for relative-error measurement (long
 * double accumulation of the stored operands).  Not a reference function. */
void or_truth_csr_f32(const int32_t* row_ptr, const int32_t* col, const float* val,
                      const float* x, const float* y0, double* y, int32_t N);
void or_truth_csr_f64(const int32_t* row_ptr, const int32_t* col, const double* val,
                      const double* x, const double* y0, double* y, int32_t N);

/* ---------------- parallel CPU baseline (reference worker partitioning) -- */
/* static_nnz: src/parallel/src/sparse32.js:2769-2821.  Fills row_start /
 * row_end (nw entries each). */
void or_static_nnz(const int32_t* row_ptr, int32_t N, int32_t nw,
                   int32_t* row_start, int32_t* row_end);
/* Parallel CSR over static_nnz ranges (src/parallel/tests/main32.js:150-313,
 * src/parallel/src/sparse_opt_32.wat:1712-1771). */
void or_par_spmv_csr_f32(int nthreads, const int32_t* row_ptr, const int32_t* col,
                         const float* val, const float* x, float* y, int32_t N);
void or_par_spmv_csr_f64(int nthreads, const int32_t* row_ptr, const int32_t* col,
                         const double* val, const double* x, double* y, int32_t N);
/* Parallel COO: nnz split, private y per worker, then nw row-split
 * reductions (src/parallel/src/sparse32.js:2637-2693,
 * src/parallel/src/sparse_opt_32.wat:1389-1481).  wy: nthreads*N scratch. */
void or_par_spmv_coo_f32(int nthreads, const int32_t* row, const int32_t* col,
                         const float* val, const float* x, float* y, int32_t N,
                         int64_t nnz, float* wy);
void or_par_spmv_coo_f64(int nthreads, const int32_t* row, const int32_t* col,
                         const double* val, const double* x, double* y, int32_t N,
                         int64_t nnz, double* wy);
/* Parallel DIA / ELL: even row split over the column-layout data, the
 * "dia_col_basic" and "ell_col" worker kernels (src/parallel/tests/main32.js:749-790,
 * :1048-1080). */
void or_par_spmv_dia_f64(int nthreads, const int32_t* offset, const double* data,
                         int32_t N, int32_t nd, int32_t stride, const double* x, double* y);
void or_par_spmv_dia_f32(int nthreads, const int32_t* offset, const float* data,
                         int32_t N, int32_t nd, int32_t stride, const float* x, float* y);
void or_par_spmv_ell_f64(int nthreads, const int32_t* indices, const double* data,
                         int32_t N, int32_t nc, const double* x, double* y);
void or_par_spmv_ell_f32(int nthreads, const int32_t* indices, const float* data,
                         int32_t N, int32_t nc, const float* x, float* y);
/* The same over the parallel build's row-by-row layout (data[i*nd + d],
 * indices[i*nc + k]): the "dia_row" / "ell_row" worker kernels
 * (src/parallel/src/sparse_opt_32.wat:8213-8269, :8292-8347). */
void or_par_spmv_dia_rows_f32(int nthreads, const int32_t* offset, const float* data, int32_t N,
                              int32_t nd, const float* x, float* y);
void or_par_spmv_dia_rows_f64(int nthreads, const int32_t* offset, const double* data, int32_t N,
                              int32_t nd, const double* x, double* y);
void or_par_spmv_ell_rows_f32(int nthreads, const int32_t* indices, const float* data, int32_t N,
                              int32_t nc, const float* x, float* y);
void or_par_spmv_ell_rows_f64(int nthreads, const int32_t* indices, const double* data, int32_t N,
                              int32_t nc, const double* x, double* y);

/* ---------------- conversions ---------------- */
/* coo_csr: src/sequential/src/sparse32.js:1674-1720 with the per-row stable
 * bubble sort `sort` :1612-1627.  val_bytes = 4 or 8. */
void or_coo_csr(int val_bytes, const int32_t* row, const int32_t* col, const void* val,
                int32_t N, int64_t nnz, int32_t* csr_row, int32_t* csr_col, void* csr_val);
/* coo_csc: src/sequential/src/sparse32.js:1629-1671. */
void or_coo_csc(int val_bytes, const int32_t* row, const int32_t* col, const void* val,
                int32_t ncols, int64_t nnz, int32_t* csc_col, int32_t* csc_row, void* csc_val);
/* num_cols: :1436-1447.  Returns max row length. */
int32_t or_num_cols(const int32_t* row_ptr, int32_t N);
/* Refusal predicate of csr_ell (:1457) and csr_dia (:1525), evaluated in
 * double precision as JS does: admit iff w*N < 2^27 and (w*N)/nnz <= 5.
 * Returns 1 when admitted. */
int or_format_admitted(int64_t width, int64_t N, int64_t nnz);
/* csr_ell fill: :1464-1484 (indices/data zero-filled, column-major). */
void or_csr_ell(int val_bytes, const int32_t* row_ptr, const int32_t* col, const void* val,
                int32_t N, int32_t nc, int32_t* indices, void* data);
/* num_diags: :1486-1512.  Returns nd; *stride = N. */
int32_t or_num_diags(const int32_t* row_ptr, const int32_t* col, int32_t N, int32_t* stride);
/* csr_dia fill: :1516-1574 (offsets ascending, last write wins). */
void or_csr_dia(int val_bytes, const int32_t* row_ptr, const int32_t* col, const void* val,
                int32_t N, int32_t nd, int32_t stride, int32_t* offset, void* data);
/* quick_sort_COO: :1577-1608 (unstable, as in the reference). */
void or_quick_sort_coo(int val_bytes, int32_t* row, int32_t* col, void* val, int64_t left,
                       int64_t right);

/* ---------------- level sets and SpTS ---------------- */
/* CSR_create_level_sets_with_reorder: src/parallel/src/sparse32.js:3010-3181
 * (level rule :3035-3055; level_ptr :3094-3108; permutation/order
 * :3110-3119; reordered CSR :3127-3138).  Returns nlevels.  level (N),
 * level_ptr (N+1 capacity), permutation (N), order (N); the reordered CSR is
 * written when new_row != NULL. */
int32_t or_level_sets(int val_bytes, const int32_t* row_ptr, const int32_t* col,
                      const void* val, int32_t N, int32_t* level, int32_t* level_ptr,
                      int32_t* permutation, int32_t* order, int32_t* new_row,
                      int32_t* new_col, void* new_val);
/* Row kernel used by the level-set and hybrid solves:
 * src/parallel/src/sparse_opt_32.wat:11679-11757.  t = 0; t += L_ij*y_j over
 * the off-diagonals in order; y_i = (b_i - t)/L_ii (diagonal stored last).
 * Rows are solved in index order, which for a level-ordered matrix gives the
 * same values as the level-by-level parallel solve (:11759-11980). */
void or_spts_csr_f32(const int32_t* row_ptr, const int32_t* col, const float* val,
                     const float* b, float* y, int32_t N);
void or_spts_csr_f64(const int32_t* row_ptr, const int32_t* col, const double* val,
                     const double* b, double* y, int32_t N);
/* Sync-free order: src/parallel/src/spts_opt_32.wat:8-117.  t = b_i;
 * t -= L_ij*y_j in order; y_i = t/L_ii. */
void or_spts_syncfree_f32(const int32_t* row_ptr, const int32_t* col, const float* val,
                          const float* b, float* y, int32_t N);
void or_spts_syncfree_f64(const int32_t* row_ptr, const int32_t* col, const double* val,
                          const double* b, double* y, int32_t N);
/* Extended-precision truth solve (not a reference function). */
void or_truth_spts(int val_bytes, const int32_t* row_ptr, const int32_t* col,
                   const void* val, const void* b, double* y, int32_t N);
/* Parallel level-set CPU baseline: level barrier + even row split per level
 * (src/parallel/src/spts_opt_32.wat:339-546), on the level-reordered matrix. */
void or_par_spts_level_f64(int nthreads, const int32_t* level_ptr, int32_t nlevels,
                           const int32_t* row_ptr, const int32_t* col, const double* val,
                           const double* b, double* y, int32_t N);
void or_par_spts_level_f32(int nthreads, const int32_t* level_ptr, int32_t nlevels,
                           const int32_t* row_ptr, const int32_t* col, const float* val,
                           const float* b, float* y, int32_t N);
/* Parallel sync-free CPU baseline: cyclic rows per worker, per-row ready
 * flags (flag[N], caller-owned), bounded spins; 0 on success, -1 when a wait
 * ran out (src/parallel/src/spts_opt_32.wat:8-260). */
int or_par_spts_syncfree_f64(int nthreads, const int32_t* row_ptr, const int32_t* col,
                             const double* val, const double* b, double* y, int32_t N,
                             int32_t* flag);
int or_par_spts_syncfree_f32(int nthreads, const int32_t* row_ptr, const int32_t* col,
                             const float* val, const float* b, float* y, int32_t N,
                             int32_t* flag);

/* ---------------- checksum ---------------- */
/* fletcher_sum: src/sequential/src/sparse32.js:1286-1311 (matlab_modulo on
 * doubles, 255 modulus, sum2*256 + sum1, parseInt). */
int64_t or_fletcher_f32(const float* y, int64_t n);
int64_t or_fletcher_f64(const double* y, int64_t n);

/* ---------------- structure operations (FP32 and FP64 values) ---------------- */
/* Nonzero test of every eliminate_zeros kernel: v > 0 || v < 0 (drops +0, -0
 * and NaN): src/sequential/src/sparse_opt_32.wat:500-521. */
int64_t or_count_nonzeros(int val_bytes, const void* val, int64_t n);
/* copy_nonzeros_coo: :523-546 (stable compaction). Returns the count. */
int64_t or_copy_nonzeros_coo(int val_bytes, const int32_t* row, const int32_t* col,
                             const void* val, int64_t nnz, int32_t* orow, int32_t* ocol,
                             void* oval);
/* copy_nonzeros_csr: :548-595 over the N rows (out_row_ptr rebuilt). */
void or_copy_nonzeros_csr(int val_bytes, const int32_t* row_ptr, const int32_t* col,
                          const void* val, int32_t N, int32_t* orow_ptr, int32_t* ocol,
                          void* oval);
/* count_nonzeros_dia :1948-2039 -> (count_diags, nnz); copy_nonzeros_dia
 * :2041-2134 packs each kept diagonal's nonzeros contiguously from the
 * diagonal's first in-band row (odata must be zero-filled, ndiags_out*stride). */
void or_count_nonzeros_dia(int val_bytes, const int32_t* offset, const void* data,
                           int32_t nd, int32_t stride, int32_t N, int32_t* count_diags,
                           int64_t* count);
void or_copy_nonzeros_dia(int val_bytes, const int32_t* offset, const void* data, int32_t nd,
                          int32_t stride, int32_t N, int32_t* ooffset, void* odata);
/* count_nonzeros_ell :5821-5893 -> (count_cols, nnz); copy_nonzeros_ell
 * :5895-5947 packs each row's nonzeros in slot order (outputs zero-filled). */
void or_count_nonzeros_ell(int val_bytes, const void* data, int32_t nc, int32_t N,
                           int32_t* count_cols, int64_t* count);
void or_copy_nonzeros_ell(int val_bytes, const void* data, const int32_t* indices, int32_t nc,
                          int32_t N, void* odata, int32_t* oindices);
/* transpose_csr :6348-6477 (counting sort by column, stable in row order). */
void or_transpose_csr(int val_bytes, const int32_t* row_ptr, const int32_t* col, const void* val,
                      int32_t N, int64_t nnz, int32_t* orow_ptr, int32_t* ocol, void* oval);
/* transpose_dia :6479-6572: offsets negated in the same order, each in-band
 * run moved to the negated diagonal's in-band rows.  Slots outside the band
 * are left as they are in odata (callers zero-fill). */
void or_transpose_dia(int val_bytes, const int32_t* offset, const void* data, int32_t nd,
                      int32_t stride, int32_t N, int32_t* ooffset, void* odata);
/* count_transpose_cols_ell :6574-6632 and transpose_ell :6634-6701 (source
 * rows outer, slots inner; odata/oindices zero-filled by the caller). */
int32_t or_count_transpose_cols_ell(int val_bytes, const void* data, const int32_t* indices,
                                    int32_t nc, int32_t N);
void or_transpose_ell(int val_bytes, const void* data, const int32_t* indices, int32_t nc,
                      int32_t N, void* odata, int32_t* oindices);

/* ---------------- element-wise maps ---------------- */
/* op codes (shared with libsparse_b200): 0 expm1, 1 log1p, 2 sin, 3 tan,
 * 4 pow(p), 5 deg2rad, 6 rad2deg, 7 sign, 8 abs, 9 neg, 10 sqrt, 11 ceil,
 * 12 floor, 13 trunc, 14 nearest, 15 multiply(p).  `kind` 0 = the COO/CSR
 * kernels (sign: v > 0 ? 1 : -1), 1 = the DIA/ELL kernels (sign: 0 -> 0).
 * f32 transcendentals are computed in double and rounded, as the imported
 * JavaScript Math functions are (src/sequential/src/sparse_opt_32.wat:5-9). */
void or_map(int val_bytes, int kind, int op, double p, const void* in, void* out, int64_t n);
/* DIA maps touch only in-band slots (src/sequential/src/sparse_opt_32.wat:2137-4976). */
void or_map_dia(int val_bytes, int op, double p, const int32_t* offset, const void* in,
                void* out, int32_t nd, int32_t stride, int32_t N);

/* spts_csc: src/sequential/src/sparse_opt_32.wat:11-148 (y = x; per column
 * j: y_j /= first entry; y_r -= L_rj*y_j for the rest of the column; the
 * 4-wide SIMD body rounds each lane like the scalar one). */
void or_spts_csc(int val_bytes, const int32_t* col_ptr, const int32_t* row, const void* val,
                 const void* x, void* y, int32_t N);

/* ---------------- COO reductions ---------------- */
/* diagonal_coo :1707-1798: the pointer walk over a row-sorted COO; diag
 * holds N - |k| slots and must be zero-filled (create_vec). */
void or_diagonal_coo(int val_bytes, int32_t k, const int32_t* row, const int32_t* col,
                     const void* val, void* diag, int32_t N, int64_t nnz);
/* min_coo :1847-1946 (axis 1; out zero-filled, as create_vec leaves it),
 * including its accumulator carried into empty rows and its early returns. */
void or_min_coo(int val_bytes, int32_t axis, const int32_t* row, const void* val, void* out,
                int32_t N, int64_t nnz);
/* Row sums in storage order (axis 1): what sum_coo :1800-1845 computes when
 * its row counter is not also advanced per entry. */
void or_sum_coo_rows(int val_bytes, int32_t axis, const int32_t* row, const void* val,
                     void* out, int32_t N, int64_t nnz);

/* ---------------- row reordering ---------------- */
/* sort_rows_by_nnz: src/parallel/src/sparse32.js:2148-2218 (stable counting
 * sort of rows by length; new CSR with rows in that order, columns kept).
 * small_rows[q] = rows with at most q nonzeros (num_zero_rows ...
 * num_three_rows). */
void or_sort_rows_by_nnz(int val_bytes, const int32_t* row_ptr, const int32_t* col,
                         const void* val, int32_t N, int32_t* nrow_ptr, int32_t* ncol,
                         void* nval, int32_t* nnz_per_row, int32_t* permutation,
                         int32_t* small_rows);
/* sort_y_rows_by_nnz :2220-2235: y_new[permutation[i]] = y[i]. */
void or_unpermute_rows(int val_bytes, const int32_t* permutation, const void* in, void* out,
                       int32_t N);
/* calculate_csr_locality_index :2238-2269. */
double or_csr_locality_index(const int32_t* row_ptr, const int32_t* col, int32_t N, int64_t nnz);
/* reorder_NN (src/parallel/src/sparse32.js:2271-2622): nearest-neighbour row
 * order by Jaccard similarity of 16-column lines, window w; walk[N] (the
 * order of input rows), perm_out[N] (composed with perm_in, NULL =
 * identity), the reordered CSR (row pointers written; the reference's are
 * not). */
void or_reorder_nn(int val_bytes, const int32_t* row_ptr, const int32_t* col, const void* val,
                   int32_t N, int w, const int32_t* perm_in, int32_t* walk, int32_t* perm_out,
                   int32_t* new_row, int32_t* new_col, void* new_val);
/* The same with the similarity list's element width chosen: list_bytes 4 is
 * the FP32 build's Float32Array (src/parallel/src/sparse32.js:2444, what
 * or_reorder_nn and the device use), 8 the FP64 build's Float64Array
 * (src/parallel/src/sparse64.js:1593). */
void or_reorder_nn_ex(int val_bytes, int list_bytes, const int32_t* row_ptr, const int32_t* col,
                      const void* val, int32_t N, int w, const int32_t* perm_in, int32_t* walk,
                      int32_t* perm_out, int32_t* new_row, int32_t* new_col, void* new_val);

/* ---------------- Matrix Market input ---------------- */
/* read_MM_header / calculate_actual_nnz / read_matrix_MM_files:
 * src/sequential/src/sparse32.js:1889-1981, on text split into lines at
 * '\n' and fields at single spaces (load_file :2454-2497).  Header: field =
 * token 3 and symmetry = token 4 of the first line; lines starting with '%'
 * skipped; then "nrows ncols nentries".  Returns 0, or -1 when nentries
 * exceeds 2^27 / the counted nnz exceeds 2^28 (the reference throws).
 * field: 0 real, 1 integer, 2 pattern, 3 complex, -1 other; symmetric = 1
 * for the symmetry token "symmetric".  The first call (row == NULL) reads
 * the header only; the second fills row/col (1-based, as in the file) and
 * val (f64; not written for pattern) and the counted nnz, including the
 * reference's fallback nnz = nentries when the count is 0. */
int or_mm_read(const char* text, int64_t len, int64_t* nrows, int64_t* ncols, int64_t* nentries,
               int32_t* field, int32_t* symmetric, int32_t* row, int32_t* col, double* val,
               int64_t* nnz);
/* create_COO_from_MM :2103-2172 (lower = 0; nnz from or_mm_read) and
 * create_LCOO_from_MM :1983-2099 (lower = 1: strictly lower entries, the
 * upper ones mirrored for "symmetric", explicit zeros dropped, then a unit
 * diagonal appended; returns its nnz), both followed by quick_sort_COO.
 * Values are stored with val_bytes (4: the Float32Array of sparse32.js,
 * 8: sparse64.js).  out arrays hold nnz entries. */
int64_t or_mm_coo(int val_bytes, int lower, int32_t field, int32_t symmetric, int64_t nrows,
                  int64_t nentries, int64_t nnz, const int32_t* row, const int32_t* col,
                  const double* val, int32_t* out_row, int32_t* out_col, void* out_val);

#ifdef __cplusplus
}
#endif
#endif
