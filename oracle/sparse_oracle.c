/*
 * sparse_oracle.c -- CPU restatement of SciWasm.Sparse's sparse kernels.
 *
 * TEST INFRASTRUCTURE ONLY (correctness oracle + timed CPU baseline); the
 * product never links it.  Parity status: the restatements of the reference's
 * WebAssembly kernels and of its JavaScript conversions, partitioner, level
 * sets, Matrix Market input and row reorderings are pinned bit for bit to
 * outputs of those functions run from their source text
 * (tests/golden/wat_vectors.npz, tests/golden/js_vectors.npz).  Each function cites the reference lines it restates; paths are
 * relative to the SciWasm.Sparse project root.  Build with
 * -O2 -ffp-contract=off -fno-fast-math so that separate mul and add are kept
 * (wasm has no fused multiply-add).
 */
#include "sparse_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include <sched.h>

/* ======================= SpMV, serial storage order ======================= */

/* spmv_coo: src/sequential/src/sparse_opt_32.wat:175-202.  For k in storage
 * order: y[row[k]] = (val[k]*x[col[k]]) + y[row[k]]. */
#define DEF_SPMV_COO(T, SFX)                                                        \
  void or_spmv_coo_##SFX(const int32_t* row, const int32_t* col, const T* val,       \
                         const T* x, T* y, int64_t nnz) {                           \
    for (int64_t k = 0; k < nnz; ++k) {                                             \
      T p = val[k] * x[col[k]];                                                     \
      y[row[k]] = p + y[row[k]];                                                    \
    }                                                                               \
  }
DEF_SPMV_COO(float, f32)
DEF_SPMV_COO(double, f64)

/* spmv_csr: src/sequential/src/sparse_opt_32.wat:227-271.  Rows without
 * entries are not written (:243 `if j < rowptr[i+1]`); otherwise
 * temp = y[i]; temp = (val*x[col]) + temp in storage order; y[i] = temp. */
#define DEF_SPMV_CSR(T, SFX)                                                        \
  void or_spmv_csr_##SFX(const int32_t* row_ptr, const int32_t* col, const T* val,   \
                         const T* x, T* y, int32_t N) {                             \
    for (int32_t i = 0; i < N; ++i) {                                               \
      int32_t j = row_ptr[i], e = row_ptr[i + 1];                                   \
      if (j < e) {                                                                  \
        T t = y[i];                                                                 \
        for (; j != e; ++j) {                                                       \
          T p = val[j] * x[col[j]];                                                 \
          t = p + t;                                                                \
        }                                                                           \
        y[i] = t;                                                                   \
      }                                                                             \
    }                                                                               \
  }
DEF_SPMV_CSR(float, f32)
DEF_SPMV_CSR(double, f64)

/* spmv_dia: src/sequential/src/sparse_opt_32.wat:290-407.  For each stored
 * diagonal d (offset k) and i in [max(0,-k), min(N, N-k)):
 * y[i] = (data[d*stride + i - move]*x[i+k]) + y[i], move = N - stride for
 * k < 0 (0 with stride = N).  The SIMD body is element-wise, so the scalar
 * loop below gives identical bits. */
#define DEF_SPMV_DIA(T, SFX)                                                        \
  void or_spmv_dia_##SFX(const int32_t* offset, const T* data, int32_t N,           \
                         int32_t nd, int32_t stride, const T* x, T* y) {            \
    for (int32_t d = 0; d < nd; ++d) {                                              \
      int32_t k = offset[d];                                                        \
      int64_t move = (k < 0) ? (int64_t)(N - stride) : 0;                           \
      int32_t n = (k < 0) ? -k : 0;                                                 \
      int32_t iend = (N < N - k) ? N : N - k;                                       \
      const T* dd = data + (int64_t)d * stride - move;                              \
      for (int32_t i = n; i < iend; ++i) {                                          \
        T p = dd[i] * x[i + k];                                                     \
        y[i] = p + y[i];                                                            \
      }                                                                             \
    }                                                                               \
  }
DEF_SPMV_DIA(float, f32)
DEF_SPMV_DIA(double, f64)

/* spmv_ell: src/sequential/src/sparse_opt_32.wat:427-479.  Column-major; all
 * nc*N slots are visited, padding (data 0, index 0) included. */
#define DEF_SPMV_ELL(T, SFX)                                                        \
  void or_spmv_ell_##SFX(const int32_t* indices, const T* data, int32_t N,          \
                         int32_t nc, const T* x, T* y) {                            \
    if (!(nc > 0 && N > 0)) return;                                                 \
    for (int32_t j = 0; j < nc; ++j) {                                              \
      const int64_t base = (int64_t)j * N;                                          \
      for (int32_t i = 0; i < N; ++i) {                                             \
        T p = data[base + i] * x[indices[base + i]];                                \
        y[i] = p + y[i];                                                            \
      }                                                                             \
    }                                                                               \
  }
DEF_SPMV_ELL(float, f32)
DEF_SPMV_ELL(double, f64)

#define DEF_TRUTH_CSR(T, SFX)                                                       \
  void or_truth_csr_##SFX(const int32_t* row_ptr, const int32_t* col, const T* val,  \
                          const T* x, const T* y0, double* y, int32_t N) {          \
    for (int32_t i = 0; i < N; ++i) {                                               \
      long double t = y0 ? (long double)y0[i] : 0.0L;                               \
      for (int32_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j)                         \
        t += (long double)val[j] * (long double)x[col[j]];                          \
      y[i] = (double)t;                                                             \
    }                                                                               \
  }
DEF_TRUTH_CSR(float, f32)
DEF_TRUTH_CSR(double, f64)

/* ======================= parallel CPU baseline ======================= */

/* static_nnz: src/parallel/src/sparse32.js:2769-2821.  Greedy contiguous
 * row ranges: each worker takes rows while its running sum is below
 * floor(rem_nnz/rem_nw).  row_end entries that the reference never assigns
 * keep the zero of a fresh Int32Array. */
void or_static_nnz(const int32_t* row_ptr, int32_t N, int32_t nw, int32_t* row_start,
                   int32_t* row_end) {
  int64_t rem_nnz = (int64_t)row_ptr[N] - row_ptr[0];
  int32_t rem_nw = nw;
  int32_t index = 0;
  int32_t i;
  for (i = 0; i < nw; ++i) { row_start[i] = 0; row_end[i] = 0; }
  for (i = 0; i < nw; ++i) {
    if (index == N) {
      row_start[i] = row_end[i] = N;
      continue;
    }
    int64_t ideal = (int64_t)floor((double)rem_nnz / (double)rem_nw);
    row_start[i] = index;
    int64_t sum = 0;
    for (int32_t j = index; j < N; ++j) {
      if (sum < ideal) {
        sum += row_ptr[j + 1] - row_ptr[j];
        index++;
      } else {
        row_end[i] = index;
        break;
      }
    }
    rem_nnz -= sum;
    rem_nw--;
  }
  row_end[i - 1] = N;
}

static int clamp_threads(int nt) { return nt < 1 ? 1 : (nt > 256 ? 256 : nt); }

/* Worker pool stand-in: nt POSIX threads, each with its id, sharing one
 * barrier, as the reference's Web Workers share one wasm memory. */
typedef struct par_job {
  int nt;
  pthread_barrier_t bar;
  void (*fn)(struct par_job*, int);
  const void* a[8];
  void* m[4];
  int64_t n[6];
} par_job;

typedef struct { par_job* job; int id; } par_arg;

static void* par_entry(void* p) {
  par_arg* a = (par_arg*)p;
  a->job->fn(a->job, a->id);
  return NULL;
}

static void par_run(par_job* job) {
  int nt = job->nt;
  pthread_t th[256];
  par_arg args[256];
  pthread_barrier_init(&job->bar, NULL, (unsigned)nt);
  for (int i = 1; i < nt; ++i) {
    args[i].job = job;
    args[i].id = i;
    pthread_create(&th[i], NULL, par_entry, &args[i]);
  }
  job->fn(job, 0);
  for (int i = 1; i < nt; ++i) pthread_join(th[i], NULL);
  pthread_barrier_destroy(&job->bar);
}

#define DEF_PAR_CSR(T, SFX)                                                         \
  static void par_csr_##SFX(par_job* j, int id) {                                   \
    const int32_t* rs = (const int32_t*)j->a[5];                                    \
    const int32_t* re = (const int32_t*)j->a[6];                                    \
    if (re[id] > rs[id])                                                            \
      or_spmv_csr_##SFX((const int32_t*)j->a[0] + rs[id], (const int32_t*)j->a[1],   \
                        (const T*)j->a[2], (const T*)j->a[3], (T*)j->m[0] + rs[id],  \
                        re[id] - rs[id]);                                           \
  }                                                                                 \
  void or_par_spmv_csr_##SFX(int nthreads, const int32_t* row_ptr,                   \
                             const int32_t* col, const T* val, const T* x, T* y,     \
                             int32_t N) {                                           \
    par_job job;                                                                    \
    job.nt = clamp_threads(nthreads);                                               \
    int32_t* rs = (int32_t*)malloc(sizeof(int32_t) * job.nt);                       \
    int32_t* re = (int32_t*)malloc(sizeof(int32_t) * job.nt);                       \
    or_static_nnz(row_ptr, N, job.nt, rs, re);                                      \
    job.fn = par_csr_##SFX;                                                         \
    job.a[0] = row_ptr; job.a[1] = col; job.a[2] = val; job.a[3] = x;               \
    job.a[5] = rs; job.a[6] = re; job.m[0] = y;                                     \
    par_run(&job);                                                                  \
    free(rs);                                                                       \
    free(re);                                                                       \
  }
DEF_PAR_CSR(float, f32)
DEF_PAR_CSR(double, f64)

/* sparse_spmv_coo: src/parallel/src/sparse32.js:2637-2693.  Worker i takes
 * nnz [i*q, (i+1)*q) (last worker + remainder) into its private w_y[i]; then
 * nw rounds of `sum` (src/parallel/src/sparse_opt_32.wat:1420-1481) add
 * w_y[0], w_y[1], ... into y, each round row-split across the workers. */
#define DEF_PAR_COO(T, SFX)                                                         \
  static void par_coo_##SFX(par_job* j, int id) {                                   \
    int nt = j->nt;                                                                 \
    int64_t nnz = j->n[0];                                                          \
    int32_t N = (int32_t)j->n[1];                                                   \
    T* y = (T*)j->m[0];                                                             \
    T* wy = (T*)j->m[1];                                                            \
    int64_t q = nnz / nt, remq = nnz - q * nt;                                      \
    int32_t npw = N / nt, remN = N - npw * nt;                                      \
    T* w = wy + (int64_t)id * N;                                                    \
    memset(w, 0, sizeof(T) * (size_t)N);                                            \
    int64_t s = id * q, e = (id + 1) * q + (id == nt - 1 ? remq : 0);               \
    or_spmv_coo_##SFX((const int32_t*)j->a[0] + s, (const int32_t*)j->a[1] + s,      \
                      (const T*)j->a[2] + s, (const T*)j->a[3], w, e - s);          \
    pthread_barrier_wait(&j->bar);                                                  \
    for (int k = 0; k < nt; ++k) {                                                  \
      const T* wk = wy + (int64_t)k * N;                                            \
      int32_t rs = id * npw, re = (id + 1) * npw + (id == nt - 1 ? remN : 0);       \
      for (int32_t r = rs; r < re; ++r) y[r] = y[r] + wk[r];                        \
      pthread_barrier_wait(&j->bar);                                                \
    }                                                                               \
  }                                                                                 \
  void or_par_spmv_coo_##SFX(int nthreads, const int32_t* row, const int32_t* col,  \
                             const T* val, const T* x, T* y, int32_t N, int64_t nnz, \
                             T* wy) {                                               \
    par_job job;                                                                    \
    job.nt = clamp_threads(nthreads);                                               \
    job.fn = par_coo_##SFX;                                                         \
    job.a[0] = row; job.a[1] = col; job.a[2] = val; job.a[3] = x;                   \
    job.m[0] = y; job.m[1] = wy; job.n[0] = nnz; job.n[1] = N;                      \
    par_run(&job);                                                                  \
  }
DEF_PAR_COO(float, f32)
DEF_PAR_COO(double, f64)

/* Row-split column-layout DIA: the "dia_col_basic" worker kernel
 * (src/parallel/tests/main32.js:749-790, src/parallel/src/sparse_opt_32.wat
 * spmv_dia_col_basic, :8991): each worker applies every diagonal to its own
 * row range, so the per-row order equals the serial one (and equals the
 * row-layout "dia_row" kernel's, :8213-8269). */
#define DEF_PAR_DIA(T, SFX)                                                         \
  static void par_dia_##SFX(par_job* j, int id) {                                   \
    int nt = j->nt;                                                                 \
    const int32_t* offset = (const int32_t*)j->a[0];                                \
    const T* data = (const T*)j->a[1];                                              \
    const T* x = (const T*)j->a[3];                                                 \
    T* y = (T*)j->m[0];                                                             \
    int32_t N = (int32_t)j->n[0], nd = (int32_t)j->n[1], stride = (int32_t)j->n[2];  \
    int32_t npw = N / nt, remN = N - npw * nt;                                      \
    int32_t s = id * npw, e = (id + 1) * npw + (id == nt - 1 ? remN : 0);           \
    for (int32_t d = 0; d < nd; ++d) {                                              \
      int32_t k = offset[d];                                                        \
      int64_t move = (k < 0) ? (int64_t)(N - stride) : 0;                           \
      int32_t lo = (k < 0) ? -k : 0;                                                \
      int32_t hi = (N < N - k) ? N : N - k;                                         \
      if (lo < s) lo = s;                                                           \
      if (hi > e) hi = e;                                                           \
      const T* dd = data + (int64_t)d * stride - move;                              \
      for (int32_t i = lo; i < hi; ++i) {                                           \
        T p = dd[i] * x[i + k];                                                     \
        y[i] = p + y[i];                                                            \
      }                                                                             \
    }                                                                               \
  }                                                                                 \
  void or_par_spmv_dia_##SFX(int nthreads, const int32_t* offset, const T* data,    \
                             int32_t N, int32_t nd, int32_t stride, const T* x,     \
                             T* y) {                                                \
    par_job job;                                                                    \
    job.nt = clamp_threads(nthreads);                                               \
    job.fn = par_dia_##SFX;                                                         \
    job.a[0] = offset; job.a[1] = data; job.a[3] = x; job.m[0] = y;                 \
    job.n[0] = N; job.n[1] = nd; job.n[2] = stride;                                 \
    par_run(&job);                                                                  \
  }
DEF_PAR_DIA(float, f32)
DEF_PAR_DIA(double, f64)

/* Row-split column-layout ELL: the "ell_col" worker kernel
 * (src/parallel/tests/main32.js:1048-1080, src/parallel/src/sparse_opt_32.wat:11055-11106). */
#define DEF_PAR_ELL(T, SFX)                                                         \
  static void par_ell_##SFX(par_job* j, int id) {                                   \
    int nt = j->nt;                                                                 \
    const int32_t* indices = (const int32_t*)j->a[0];                               \
    const T* data = (const T*)j->a[1];                                              \
    const T* x = (const T*)j->a[3];                                                 \
    T* y = (T*)j->m[0];                                                             \
    int32_t N = (int32_t)j->n[0], nc = (int32_t)j->n[1];                            \
    int32_t npw = N / nt, remN = N - npw * nt;                                      \
    int32_t s = id * npw, e = (id + 1) * npw + (id == nt - 1 ? remN : 0);           \
    for (int32_t c = 0; c < nc; ++c) {                                              \
      const int64_t base = (int64_t)c * N;                                          \
      for (int32_t i = s; i < e; ++i) {                                             \
        T p = data[base + i] * x[indices[base + i]];                                \
        y[i] = p + y[i];                                                            \
      }                                                                             \
    }                                                                               \
  }                                                                                 \
  void or_par_spmv_ell_##SFX(int nthreads, const int32_t* indices, const T* data,   \
                             int32_t N, int32_t nc, const T* x, T* y) {             \
    par_job job;                                                                    \
    job.nt = clamp_threads(nthreads);                                               \
    job.fn = par_ell_##SFX;                                                         \
    job.a[0] = indices; job.a[1] = data; job.a[3] = x; job.m[0] = y;                \
    job.n[0] = N; job.n[1] = nc;                                                    \
    par_run(&job);                                                                  \
  }
DEF_PAR_ELL(float, f32)
DEF_PAR_ELL(double, f64)

/* Row-split row-layout DIA and ELL: the "dia_row" and "ell_row" worker
 * kernels (src/parallel/tests/main32.js:688-694 and the ELL dispatch beside
 * it; src/parallel/src/sparse_opt_32.wat:8213-8269 spmv_dia and :8292-8347
 * spmv_ell), over the parallel build's row-by-row data (data[i*nd + d],
 * src/parallel/src/sparse32.js csr_dia / csr_ell).  Per row: t = y_i; for
 * each slot in order, t = v*x + t (DIA: only while the column is in range;
 * ELL: until a negative index); y_i = t.  The same per-row order as the
 * column-layout kernels above. */
#define DEF_PAR_ROWS(T, SFX)                                                        \
  static void par_dia_rows_##SFX(par_job* j, int id) {                              \
    int nt = j->nt;                                                                 \
    const int32_t* offset = (const int32_t*)j->a[0];                                \
    const T* data = (const T*)j->a[1];                                              \
    const T* x = (const T*)j->a[3];                                                 \
    T* y = (T*)j->m[0];                                                             \
    int32_t N = (int32_t)j->n[0], nd = (int32_t)j->n[1];                            \
    int32_t npw = N / nt, remN = N - npw * nt;                                      \
    int32_t s = id * npw, e = (id + 1) * npw + (id == nt - 1 ? remN : 0);           \
    for (int32_t i = s; i < e; ++i) {                                               \
      const T* row = data + (int64_t)i * nd;                                        \
      T t = y[i];                                                                   \
      for (int32_t d = 0; d < nd; ++d) {                                            \
        const int32_t c = i + offset[d];                                            \
        if (c >= 0 && c < N) {                                                      \
          T p = row[d] * x[c];                                                      \
          t = p + t;                                                                \
        }                                                                           \
      }                                                                             \
      y[i] = t;                                                                     \
    }                                                                               \
  }                                                                                 \
  void or_par_spmv_dia_rows_##SFX(int nthreads, const int32_t* offset, const T* data, \
                                  int32_t N, int32_t nd, const T* x, T* y) {        \
    par_job job;                                                                    \
    job.nt = clamp_threads(nthreads);                                               \
    job.fn = par_dia_rows_##SFX;                                                    \
    job.a[0] = offset; job.a[1] = data; job.a[3] = x; job.m[0] = y;                 \
    job.n[0] = N; job.n[1] = nd;                                                    \
    par_run(&job);                                                                  \
  }                                                                                 \
  static void par_ell_rows_##SFX(par_job* j, int id) {                              \
    int nt = j->nt;                                                                 \
    const int32_t* indices = (const int32_t*)j->a[0];                               \
    const T* data = (const T*)j->a[1];                                              \
    const T* x = (const T*)j->a[3];                                                 \
    T* y = (T*)j->m[0];                                                             \
    int32_t N = (int32_t)j->n[0], nc = (int32_t)j->n[1];                            \
    int32_t npw = N / nt, remN = N - npw * nt;                                      \
    int32_t s = id * npw, e = (id + 1) * npw + (id == nt - 1 ? remN : 0);           \
    for (int32_t i = s; i < e; ++i) {                                               \
      const int64_t base = (int64_t)i * nc;                                         \
      T t = y[i];                                                                   \
      for (int32_t k = 0; k < nc; ++k) {                                            \
        const int32_t c = indices[base + k];                                        \
        if (c < 0) break;                                                           \
        T p = data[base + k] * x[c];                                                \
        t = p + t;                                                                  \
      }                                                                             \
      y[i] = t;                                                                     \
    }                                                                               \
  }                                                                                 \
  void or_par_spmv_ell_rows_##SFX(int nthreads, const int32_t* indices, const T* data, \
                                  int32_t N, int32_t nc, const T* x, T* y) {        \
    par_job job;                                                                    \
    job.nt = clamp_threads(nthreads);                                               \
    job.fn = par_ell_rows_##SFX;                                                    \
    job.a[0] = indices; job.a[1] = data; job.a[3] = x; job.m[0] = y;                \
    job.n[0] = N; job.n[1] = nc;                                                    \
    par_run(&job);                                                                  \
  }
DEF_PAR_ROWS(float, f32)
DEF_PAR_ROWS(double, f64)

/* ======================= conversions ======================= */

static void swap_bytes(void* a, int64_t i, int64_t j, int w) {
  if (w == 4) {
    uint32_t* p = (uint32_t*)a;
    uint32_t t = p[i]; p[i] = p[j]; p[j] = t;
  } else {
    uint64_t* p = (uint64_t*)a;
    uint64_t t = p[i]; p[i] = p[j]; p[j] = t;
  }
}

static void copy_elem(void* dst, int64_t i, const void* src, int64_t j, int w) {
  if (w == 4) ((uint32_t*)dst)[i] = ((const uint32_t*)src)[j];
  else ((uint64_t*)dst)[i] = ((const uint64_t*)src)[j];
}

/* sort: src/sequential/src/sparse32.js:1612-1627.  Bubble sort of
 * array1[start, end) with array2 carried along; strict '>' keeps it stable. */
static void bubble_sort(int64_t start, int64_t end, int32_t* a1, void* a2, int w) {
  int64_t n = end - start;
  for (int64_t i = 0; i < n - 1; ++i) {
    for (int64_t j = start; j < end - i - 1; ++j) {
      if (a1[j] > a1[j + 1]) {
        int32_t t = a1[j]; a1[j] = a1[j + 1]; a1[j + 1] = t;
        swap_bytes(a2, j, j + 1, w);
      }
    }
  }
}

/* coo_csr: src/sequential/src/sparse32.js:1674-1720. */
void or_coo_csr(int w, const int32_t* row, const int32_t* col, const void* val, int32_t N,
                int64_t nnz, int32_t* csr_row, int32_t* csr_col, void* csr_val) {
  memset(csr_row, 0, sizeof(int32_t) * ((size_t)N + 1));
  for (int64_t i = 0; i < nnz; ++i) csr_row[row[i]]++;
  int32_t j = 0, j0;
  for (int32_t i = 0; i < N; ++i) {
    j0 = csr_row[i];
    csr_row[i] = j;
    j += j0;
  }
  for (int64_t i = 0; i < nnz; ++i) {
    int32_t p = csr_row[row[i]];
    csr_col[p] = col[i];
    copy_elem(csr_val, p, val, i, w);
    csr_row[row[i]]++;
  }
  for (int32_t i = N - 1; i > 0; --i) csr_row[i] = csr_row[i - 1];
  csr_row[0] = 0;
  csr_row[N] = (int32_t)nnz;
  for (int32_t i = 0; i < N; ++i) bubble_sort(csr_row[i], csr_row[i + 1], csr_col, csr_val, w);
}

/* coo_csc: src/sequential/src/sparse32.js:1629-1671 (same shape with the
 * roles of row and col exchanged). */
void or_coo_csc(int w, const int32_t* row, const int32_t* col, const void* val,
                int32_t ncols, int64_t nnz, int32_t* csc_col, int32_t* csc_row,
                void* csc_val) {
  or_coo_csr(w, col, row, val, ncols, nnz, csc_col, csc_row, csc_val);
}

/* num_cols: src/sequential/src/sparse32.js:1436-1447. */
int32_t or_num_cols(const int32_t* row_ptr, int32_t N) {
  int32_t mx = 0;
  for (int32_t i = 0; i < N; ++i) {
    int32_t t = row_ptr[i + 1] - row_ptr[i];
    if (mx < t) mx = t;
  }
  return mx;
}

/* The admission test of csr_ell (:1457) and csr_dia (:1525), in doubles.
 * nnz == 0 gives 0/0 = NaN, and NaN <= 5 is false: refused. */
int or_format_admitted(int64_t width, int64_t N, int64_t nnz) {
  double wn = (double)width * (double)N;
  double ratio = wn / (double)nnz;
  return (wn < 134217728.0) && (ratio <= 5.0);
}

/* csr_ell: src/sequential/src/sparse32.js:1464-1484. */
void or_csr_ell(int w, const int32_t* row_ptr, const int32_t* col, const void* val,
                int32_t N, int32_t nc, int32_t* indices, void* data) {
  size_t slots = (size_t)nc * (size_t)N;
  memset(indices, 0, sizeof(int32_t) * slots);
  memset(data, 0, (size_t)w * slots);
  for (int32_t i = 0; i < N; ++i) {
    int64_t k = 0;
    for (int32_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j) {
      copy_elem(data, k * N + i, val, j, w);
      indices[k * N + i] = col[j];
      k++;
    }
  }
}

/* num_diags: src/sequential/src/sparse32.js:1486-1512.  Diagonal c - i maps
 * to ind[N + c - i - 1]; stride is N. */
int32_t or_num_diags(const int32_t* row_ptr, const int32_t* col, int32_t N, int32_t* stride) {
  int32_t nd = 0;
  if (N <= 0) { *stride = N; return 0; }
  int32_t* ind = (int32_t*)calloc((size_t)2 * N - 1, sizeof(int32_t));
  for (int32_t i = 0; i < N; ++i)
    for (int32_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j)
      if (!ind[(int64_t)N + col[j] - i - 1]++) nd++;
  free(ind);
  *stride = N;
  return nd;
}

/* csr_dia: src/sequential/src/sparse32.js:1516-1574.  Offsets are the present
 * diagonals in ascending order; each entry is placed by a linear search over
 * the offsets, so a later duplicate (i, c) overwrites an earlier one. */
void or_csr_dia(int w, const int32_t* row_ptr, const int32_t* col, const void* val,
                int32_t N, int32_t nd, int32_t stride, int32_t* offset, void* data) {
  memset(data, 0, (size_t)w * (size_t)nd * (size_t)stride);
  if (N <= 0) return;
  int32_t* ind = (int32_t*)calloc((size_t)2 * N - 1, sizeof(int32_t));
  for (int32_t i = 0; i < N; ++i)
    for (int32_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j) ind[(int64_t)N + col[j] - i - 1]++;
  int32_t diag_no = -((2 * N - 1) / 2);
  int32_t index = 0;
  for (int64_t i = 0; i < 2 * (int64_t)N - 1; ++i) {
    if (ind[i]) offset[index++] = diag_no;
    diag_no++;
  }
  free(ind);
  for (int32_t i = 0; i < N; ++i) {
    for (int32_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j) {
      int32_t c = col[j];
      for (int32_t k = 0; k < nd; ++k) {
        int64_t move = 0;
        if (c - i == offset[k]) {
          if (offset[k] < 0) move = (int64_t)N - stride;
          copy_elem(data, (int64_t)k * stride + i - move, val, j, w);
          break;
        }
      }
    }
  }
}

/* quick_sort_COO: src/sequential/src/sparse32.js:1577-1608 (Hoare partition
 * on the middle element, keyed by (row, col); not stable). */
void or_quick_sort_coo(int w, int32_t* row, int32_t* col, void* val, int64_t left,
                       int64_t right) {
  while (left < right) {
    int64_t i = left, j = right;
    int64_t mid = (left + right) / 2;
    int32_t pivot = row[mid], pivot_col = col[mid];
    while (i <= j) {
      while (row[i] < pivot || (row[i] == pivot && col[i] < pivot_col)) i++;
      while (row[j] > pivot || (row[j] == pivot && col[j] > pivot_col)) j--;
      if (i <= j) {
        int32_t t = row[i]; row[i] = row[j]; row[j] = t;
        t = col[i]; col[i] = col[j]; col[j] = t;
        swap_bytes(val, i, j, w);
        i++;
        j--;
      }
    }
    /* recurse into the smaller side, loop on the larger (same result as the
     * reference's two recursive calls, bounded stack) */
    if (j - left < right - i) {
      if (left < j) or_quick_sort_coo(w, row, col, val, left, j);
      left = i;
    } else {
      if (i < right) or_quick_sort_coo(w, row, col, val, i, right);
      right = j;
    }
  }
}

/* ======================= level sets and SpTS ======================= */

/* CSR_create_level_sets_with_reorder: src/parallel/src/sparse32.js:3010-3181.
 * level[i] = 0 when row i holds exactly one entry; otherwise 1 + the maximum
 * (initialised at 0) of level[col] over all entries but the last, where rows
 * not yet visited (col >= i) still read 0.  An empty row therefore gets
 * level 1.  Rows are stably counting-sorted by level. */
int32_t or_level_sets(int w, const int32_t* row_ptr, const int32_t* col, const void* val,
                      int32_t N, int32_t* level, int32_t* level_ptr, int32_t* permutation,
                      int32_t* order, int32_t* new_row, int32_t* new_col, void* new_val) {
  int32_t max_level = 0;
  memset(level, 0, sizeof(int32_t) * (size_t)N);
  for (int32_t i = 0; i < N; ++i) {
    int32_t len = row_ptr[i + 1] - row_ptr[i];
    if (len == 1) {
      level[i] = 0;
    } else {
      int32_t m = 0;
      for (int32_t j = row_ptr[i]; j < row_ptr[i + 1] - 1; ++j)
        if (level[col[j]] > m) m = level[col[j]];
      level[i] = 1 + m;
      if (level[i] > max_level) max_level = level[i];
    }
  }
  int32_t nlev = max_level + 1;
  int32_t* freq = (int32_t*)calloc((size_t)nlev, sizeof(int32_t));
  int32_t* start = (int32_t*)calloc((size_t)nlev, sizeof(int32_t));
  for (int32_t i = 0; i < N; ++i) freq[level[i]]++;
  level_ptr[0] = 0;
  start[0] = 0;
  for (int32_t l = 1; l < nlev; ++l) start[l] = level_ptr[l] = level_ptr[l - 1] + freq[l - 1];
  level_ptr[nlev] = level_ptr[nlev - 1] + freq[nlev - 1];
  for (int32_t i = 0; i < N; ++i) {
    permutation[start[level[i]]] = i;
    order[i] = start[level[i]];
    start[level[i]]++;
  }
  free(freq);
  free(start);
  if (new_row) {
    int64_t j = 0;
    new_row[0] = 0;
    for (int32_t i = 0; i < N; ++i) {
      int32_t p = permutation[i];
      int32_t k = row_ptr[p];
      int32_t t = row_ptr[p + 1] - row_ptr[p];
      new_row[i + 1] = new_row[i] + t;
      while (t != 0) {
        new_col[j] = order[col[k]];
        copy_elem(new_val, j, val, k, w);
        j++;
        k++;
        t--;
      }
    }
  }
  return nlev;
}

/* spts_csr row kernel: src/parallel/src/sparse_opt_32.wat:11679-11757. */
#define DEF_SPTS_CSR(T, SFX)                                                        \
  void or_spts_csr_##SFX(const int32_t* row_ptr, const int32_t* col, const T* val,   \
                         const T* b, T* y, int32_t N) {                             \
    for (int32_t i = 0; i < N; ++i) {                                               \
      int32_t j = row_ptr[i], end = row_ptr[i + 1] - 1;                             \
      if (end > j) {                                                                \
        T t = (T)0;                                                                 \
        for (; j != end; ++j) {                                                     \
          T p = val[j] * y[col[j]];                                                 \
          t = t + p;                                                                \
        }                                                                           \
        y[i] = (b[i] - t) / val[end];                                               \
      } else {                                                                      \
        y[i] = b[i] / val[end];                                                     \
      }                                                                             \
    }                                                                               \
  }
DEF_SPTS_CSR(float, f32)
DEF_SPTS_CSR(double, f64)

/* spts_csr_sync_free: src/parallel/src/spts_opt_32.wat:8-117 (x aliases y,
 * pre-copied from b). */
#define DEF_SPTS_SF(T, SFX)                                                         \
  void or_spts_syncfree_##SFX(const int32_t* row_ptr, const int32_t* col,            \
                              const T* val, const T* b, T* y, int32_t N) {          \
    for (int32_t i = 0; i < N; ++i) y[i] = b[i];                                    \
    for (int32_t i = 0; i < N; ++i) {                                               \
      int32_t j = row_ptr[i] + 1, end = row_ptr[i + 1];                             \
      if (end > j) {                                                                \
        T t = y[i];                                                                 \
        int32_t k = row_ptr[i];                                                     \
        for (; k != end - 1; ++k) {                                                 \
          T p = val[k] * y[col[k]];                                                 \
          t = t - p;                                                                \
        }                                                                           \
        y[i] = t / val[end - 1];                                                    \
      } else {                                                                      \
        y[i] = y[i] / val[row_ptr[i]];                                              \
      }                                                                             \
    }                                                                               \
  }
DEF_SPTS_SF(float, f32)
DEF_SPTS_SF(double, f64)

void or_truth_spts(int w, const int32_t* row_ptr, const int32_t* col, const void* val,
                   const void* b, double* y, int32_t N) {
  long double* t = (long double*)malloc(sizeof(long double) * (size_t)(N > 0 ? N : 1));
  for (int32_t i = 0; i < N; ++i) {
    int32_t s = row_ptr[i], e = row_ptr[i + 1] - 1;
    long double acc = 0.0L;
    for (int32_t j = s; j < e; ++j) {
      long double v = (w == 4) ? (long double)((const float*)val)[j]
                               : (long double)((const double*)val)[j];
      acc += v * t[col[j]];
    }
    long double bi = (w == 4) ? (long double)((const float*)b)[i]
                              : (long double)((const double*)b)[i];
    long double d = (w == 4) ? (long double)((const float*)val)[e]
                             : (long double)((const double*)val)[e];
    t[i] = (bi - acc) / d;
    y[i] = (double)t[i];
  }
  free(t);
}

/* spts_level_csr: src/parallel/src/spts_opt_32.wat:339-546 and
 * src/parallel/src/sparse_opt_32.wat:11759-11980.  Per level, rows
 * [level_ptr[l], level_ptr[l+1]) are split len = nrows/nt with the first
 * nrows%nt workers taking one more; a barrier follows every level. */
#define DEF_PAR_SPTS(T, SFX)                                                        \
  static void par_spts_##SFX(par_job* jb, int id) {                                 \
    int nt = jb->nt;                                                                \
    const int32_t* level_ptr = (const int32_t*)jb->a[0];                            \
    const int32_t* row_ptr = (const int32_t*)jb->a[1];                              \
    const int32_t* col = (const int32_t*)jb->a[2];                                  \
    const T* val = (const T*)jb->a[3];                                              \
    const T* b = (const T*)jb->a[4];                                                \
    T* y = (T*)jb->m[0];                                                            \
    int32_t nlevels = (int32_t)jb->n[0];                                            \
    for (int32_t l = 0; l < nlevels; ++l) {                                         \
      int32_t nrows = level_ptr[l + 1] - level_ptr[l];                              \
      int32_t len = nrows / nt, rem = nrows % nt, s;                                \
      if (len != 0) {                                                               \
        if (rem > id) { s = level_ptr[l] + id * len + id; len++; }                  \
        else s = level_ptr[l] + id * len + rem;                                     \
      } else {                                                                      \
        len = (nrows > id) ? 1 : 0;                                                 \
        s = level_ptr[l] + id;                                                      \
      }                                                                             \
      for (int32_t i = s; i < s + len; ++i) {                                       \
        int32_t j = row_ptr[i], end = row_ptr[i + 1] - 1;                           \
        if (end > j) {                                                              \
          T t = (T)0;                                                               \
          for (; j != end; ++j) {                                                   \
            T p = val[j] * y[col[j]];                                               \
            t = t + p;                                                              \
          }                                                                         \
          y[i] = (b[i] - t) / val[end];                                             \
        } else {                                                                    \
          y[i] = b[i] / val[end];                                                   \
        }                                                                           \
      }                                                                             \
      pthread_barrier_wait(&jb->bar);                                               \
    }                                                                               \
  }                                                                                 \
  void or_par_spts_level_##SFX(int nthreads, const int32_t* level_ptr,              \
                               int32_t nlevels, const int32_t* row_ptr,             \
                               const int32_t* col, const T* val, const T* b, T* y,  \
                               int32_t N) {                                         \
    par_job job;                                                                    \
    (void)N;                                                                        \
    job.nt = clamp_threads(nthreads);                                               \
    job.fn = par_spts_##SFX;                                                        \
    job.a[0] = level_ptr; job.a[1] = row_ptr; job.a[2] = col; job.a[3] = val;       \
    job.a[4] = b; job.m[0] = y; job.n[0] = nlevels;                                 \
    par_run(&job);                                                                  \
  }
DEF_PAR_SPTS(float, f32)
DEF_PAR_SPTS(double, f64)

/* spts_csr_sync_free + its wrapper: src/parallel/src/spts_opt_32.wat:8-260.
 * Each worker copies its share of b into y and clears its share of the ready
 * flags; after a barrier, worker id takes rows id, id + nt, ... in order:
 * t = y[i], then for every off-diagonal (in storage order) it waits until
 * flag[col] == 1 and subtracts val * y[col]; y[i] = t / diagonal (stored
 * last), then flag[i] = 1.  Rows always wait on smaller rows, which their
 * owners reach in increasing order, so the lowest unsolved row can always
 * proceed.  The spins are bounded here (the reference's are not): a wait that
 * runs out sets the job's error word and the worker stops; the caller gets
 * -1.  Same arithmetic per row as or_spts_syncfree (bit-identical). */
#define SF_SPIN_LIMIT (1LL << 34)
#define DEF_PAR_SF(T, SFX)                                                          \
  static void par_sf_##SFX(par_job* jb, int id) {                                   \
    const int nt = jb->nt;                                                          \
    const int32_t* row_ptr = (const int32_t*)jb->a[0];                              \
    const int32_t* col = (const int32_t*)jb->a[1];                                  \
    const T* val = (const T*)jb->a[2];                                              \
    const T* b = (const T*)jb->a[3];                                                \
    T* y = (T*)jb->m[0];                                                            \
    int32_t* flag = (int32_t*)jb->m[1];                                             \
    int32_t* err = (int32_t*)jb->m[2];                                              \
    const int32_t N = (int32_t)jb->n[0];                                            \
    const int32_t npw = N / nt, remN = N - npw * nt;                                \
    const int32_t s0 = id * npw, e0 = (id + 1) * npw + (id == nt - 1 ? remN : 0);   \
    for (int32_t i = s0; i < e0; ++i) {                                             \
      y[i] = b[i];                                                                  \
      __atomic_store_n(&flag[i], 0, __ATOMIC_RELAXED);                              \
    }                                                                               \
    pthread_barrier_wait(&jb->bar);                                                 \
    for (int32_t i = id; i < N; i += nt) {                                          \
      const int32_t s = row_ptr[i], end = row_ptr[i + 1];                           \
      T t = y[i];                                                                   \
      for (int32_t k = s; k < end - 1; ++k) {                                       \
        const int32_t c = col[k];                                                   \
        int64_t spins = 0;                                                          \
        while (__atomic_load_n(&flag[c], __ATOMIC_ACQUIRE) != 1) {                  \
          if (__atomic_load_n(err, __ATOMIC_RELAXED) || ++spins > SF_SPIN_LIMIT) {  \
            __atomic_store_n(err, 1, __ATOMIC_RELAXED);                             \
            return;                                                                 \
          }                                                                         \
          if ((spins & 1023) == 0) sched_yield();                                   \
        }                                                                           \
        T p = val[k] * y[c];                                                        \
        t = t - p;                                                                  \
      }                                                                             \
      y[i] = t / val[end - 1];                                                      \
      __atomic_store_n(&flag[i], 1, __ATOMIC_RELEASE);                              \
    }                                                                               \
  }                                                                                 \
  int or_par_spts_syncfree_##SFX(int nthreads, const int32_t* row_ptr,              \
                                 const int32_t* col, const T* val, const T* b, T* y, \
                                 int32_t N, int32_t* flag) {                        \
    par_job job;                                                                    \
    int32_t err = 0;                                                                \
    job.nt = clamp_threads(nthreads);                                               \
    job.fn = par_sf_##SFX;                                                          \
    job.a[0] = row_ptr; job.a[1] = col; job.a[2] = val; job.a[3] = b;               \
    job.m[0] = y; job.m[1] = flag; job.m[2] = &err; job.n[0] = N;                   \
    par_run(&job);                                                                  \
    return err ? -1 : 0;                                                            \
  }
DEF_PAR_SF(float, f32)
DEF_PAR_SF(double, f64)

/* ======================= checksum ======================= */

/* matlab_modulo / fletcher_sum / fletcher_sum_y:
 * src/sequential/src/sparse32.js:1286-1311. */
static double matlab_modulo(double x, double y) {
  double n = floor(x / y);
  return x - n * y;
}

#define DEF_FLETCHER(T, SFX)                                                        \
  int64_t or_fletcher_##SFX(const T* y, int64_t n) {                                \
    double s1 = 0.0, s2 = 0.0;                                                      \
    for (int64_t i = 0; i < n; ++i) {                                               \
      s1 = matlab_modulo(s1 + (double)y[i], 255.0);                                 \
      s2 = matlab_modulo(s2 + s1, 255.0);                                           \
    }                                                                               \
    double r = s2 * 256.0 + s1;                                                     \
    return (int64_t)r; /* parseInt truncates toward zero */                         \
  }
DEF_FLETCHER(float, f32)
DEF_FLETCHER(double, f64)

/* ======================= structure operations ======================= */

static int is_nz(const void* a, int64_t i, int w) {
  if (w == 4) { float v = ((const float*)a)[i]; return v > 0.0f || v < 0.0f; }
  double v = ((const double*)a)[i];
  return v > 0.0 || v < 0.0;
}

int64_t or_count_nonzeros(int w, const void* val, int64_t n) {
  int64_t c = 0;
  for (int64_t i = 0; i < n; ++i) c += is_nz(val, i, w);
  return c;
}

int64_t or_copy_nonzeros_coo(int w, const int32_t* row, const int32_t* col, const void* val,
                             int64_t nnz, int32_t* orow, int32_t* ocol, void* oval) {
  int64_t o = 0;
  for (int64_t i = 0; i < nnz; ++i) {
    if (is_nz(val, i, w)) {
      orow[o] = row[i];
      ocol[o] = col[i];
      copy_elem(oval, o, val, i, w);
      o++;
    }
  }
  return o;
}

void or_copy_nonzeros_csr(int w, const int32_t* row_ptr, const int32_t* col, const void* val,
                          int32_t N, int32_t* orow_ptr, int32_t* ocol, void* oval) {
  int64_t o = 0;
  orow_ptr[0] = 0;
  for (int32_t i = 0; i < N; ++i) {
    for (int32_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j) {
      if (is_nz(val, j, w)) {
        ocol[o] = col[j];
        copy_elem(oval, o, val, j, w);
        o++;
      }
    }
    orow_ptr[i + 1] = (int32_t)o;
  }
}

static void dia_range(int32_t k, int32_t N, int32_t* lo, int32_t* hi) {
  *lo = k < 0 ? -k : 0;
  *hi = (N < N - k) ? N : N - k;
}

void or_count_nonzeros_dia(int w, const int32_t* offset, const void* data, int32_t nd,
                           int32_t stride, int32_t N, int32_t* count_diags, int64_t* count) {
  int32_t cd = 0;
  int64_t nz = 0;
  for (int32_t d = 0; d < nd; ++d) {
    int32_t lo, hi;
    dia_range(offset[d], N, &lo, &hi);
    int64_t base = (int64_t)d * stride - (offset[d] < 0 ? (int64_t)(N - stride) : 0);
    int64_t c = 0;
    for (int32_t n = lo; n < hi; ++n) c += is_nz(data, base + n, w);
    if (c) { cd++; nz += c; }
  }
  *count_diags = cd;
  *count = nz;
}

void or_copy_nonzeros_dia(int w, const int32_t* offset, const void* data, int32_t nd,
                          int32_t stride, int32_t N, int32_t* ooffset, void* odata) {
  int64_t j = 0; /* kept diagonals * stride */
  int32_t od = 0;
  for (int32_t d = 0; d < nd; ++d) {
    int32_t lo, hi;
    dia_range(offset[d], N, &lo, &hi);
    int64_t base = (int64_t)d * stride - (offset[d] < 0 ? (int64_t)(N - stride) : 0);
    int64_t out = j + lo, c = 0;
    for (int32_t n = lo; n < hi; ++n) {
      if (is_nz(data, base + n, w)) {
        copy_elem(odata, out++, data, base + n, w);
        c++;
      }
    }
    if (c) {
      ooffset[od++] = offset[d];
      j += stride;
    }
  }
}

void or_count_nonzeros_ell(int w, const void* data, int32_t nc, int32_t N, int32_t* count_cols,
                           int64_t* count) {
  int32_t* per = (int32_t*)calloc((size_t)(N > 0 ? N : 1), sizeof(int32_t));
  int32_t cc = 0;
  int64_t nz = 0;
  for (int32_t k = 0; k < nc; ++k)
    for (int32_t i = 0; i < N; ++i)
      if (is_nz(data, (int64_t)k * N + i, w)) {
        per[i]++;
        if (per[i] > cc) cc = per[i];
        nz++;
      }
  free(per);
  *count_cols = cc;
  *count = nz;
}

void or_copy_nonzeros_ell(int w, const void* data, const int32_t* indices, int32_t nc, int32_t N,
                          void* odata, int32_t* oindices) {
  int64_t* pos = (int64_t*)calloc((size_t)(N > 0 ? N : 1), sizeof(int64_t));
  for (int32_t k = 0; k < nc; ++k)
    for (int32_t i = 0; i < N; ++i) {
      int64_t s = (int64_t)k * N + i;
      if (is_nz(data, s, w)) {
        copy_elem(odata, pos[i] + i, data, s, w);
        oindices[pos[i] + i] = indices[s];
        pos[i] += N;
      }
    }
  free(pos);
}

void or_transpose_csr(int w, const int32_t* row_ptr, const int32_t* col, const void* val,
                      int32_t N, int64_t nnz, int32_t* orow_ptr, int32_t* ocol, void* oval) {
  memset(orow_ptr, 0, sizeof(int32_t) * ((size_t)N + 1));
  for (int64_t j = 0; j < nnz; ++j) orow_ptr[col[j]]++;
  int32_t sum = 0;
  for (int32_t i = 0; i < N; ++i) {
    int32_t c = orow_ptr[i];
    orow_ptr[i] = sum;
    sum += c;
  }
  orow_ptr[N] = (int32_t)nnz;
  for (int32_t i = 0; i < N; ++i)
    for (int32_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j) {
      int32_t a = orow_ptr[col[j]]++;
      ocol[a] = i;
      copy_elem(oval, a, val, j, w);
    }
  sum = 0;
  for (int32_t i = 0; i <= N; ++i) {
    int32_t t = orow_ptr[i];
    orow_ptr[i] = sum;
    sum = t;
  }
}

void or_transpose_dia(int w, const int32_t* offset, const void* data, int32_t nd, int32_t stride,
                      int32_t N, int32_t* ooffset, void* odata) {
  for (int32_t d = 0; d < nd; ++d) {
    int32_t k = offset[d];
    int32_t lo, hi;
    dia_range(k, N, &lo, &hi);
    ooffset[d] = -k;
    int32_t olo, ohi;
    dia_range(-k, N, &olo, &ohi);
    int64_t ib = (int64_t)d * stride - (k < 0 ? (int64_t)(N - stride) : 0);
    int64_t ob = (int64_t)d * stride - (-k < 0 ? (int64_t)(N - stride) : 0);
    for (int32_t t = 0; t < hi - lo; ++t) copy_elem(odata, ob + olo + t, data, ib + lo + t, w);
  }
}

int32_t or_count_transpose_cols_ell(int w, const void* data, const int32_t* indices, int32_t nc,
                                    int32_t N) {
  int32_t* cnt = (int32_t*)calloc((size_t)(N > 0 ? N : 1), sizeof(int32_t));
  int32_t cc = 0;
  for (int32_t k = 0; k < nc; ++k)
    for (int32_t i = 0; i < N; ++i) {
      int64_t s = (int64_t)k * N + i;
      if (is_nz(data, s, w)) {
        int32_t c = ++cnt[indices[s]];
        if (c > cc) cc = c;
      }
    }
  free(cnt);
  return cc;
}

void or_transpose_ell(int w, const void* data, const int32_t* indices, int32_t nc, int32_t N,
                      void* odata, int32_t* oindices) {
  int64_t* pos = (int64_t*)calloc((size_t)(N > 0 ? N : 1), sizeof(int64_t));
  for (int32_t j = 0; j < N; ++j)
    for (int32_t k = 0; k < nc; ++k) {
      int64_t s = (int64_t)k * N + j;
      if (is_nz(data, s, w)) {
        int32_t c = indices[s];
        copy_elem(odata, pos[c] + c, data, s, w);
        oindices[pos[c] + c] = j;
        pos[c] += N;
      }
    }
  free(pos);
}

/* ======================= element-wise maps ======================= */

static double map_f64(int kind, int op, double p, double v) {
  switch (op) {
    case 0: return expm1(v);
    case 1: return log1p(v);
    case 2: return sin(v);
    case 3: return tan(v);
    case 4: return pow(v, p);
    case 5: return v * (p / 180.0);
    case 6: return v / (p / 180.0);
    case 7:
      if (kind == 1 && v == 0.0) return 0.0;
      return v > 0.0 ? 1.0 : -1.0;
    case 8: return fabs(v);
    case 9: return -v;
    case 10: return sqrt(v);
    case 11: return ceil(v);
    case 12: return floor(v);
    case 13: return trunc(v);
    case 14: return nearbyint(v); /* default rounding mode: ties to even */
    case 15: return v * p;
  }
  return v;
}

static float map_f32(int kind, int op, float p, float v) {
  switch (op) {
    case 0: return (float)expm1((double)v);
    case 1: return (float)log1p((double)v);
    case 2: return (float)sin((double)v);
    case 3: return (float)tan((double)v);
    case 4: return (float)pow((double)v, (double)p);
    case 5: { float k = p / 180.0f; return v * k; }
    case 6: { float k = p / 180.0f; return v / k; }
    case 7:
      if (kind == 1 && v == 0.0f) return 0.0f;
      return v > 0.0f ? 1.0f : -1.0f;
    case 8: return fabsf(v);
    case 9: return -v;
    case 10: return sqrtf(v);
    case 11: return ceilf(v);
    case 12: return floorf(v);
    case 13: return truncf(v);
    case 14: return nearbyintf(v);
    case 15: return v * p;
  }
  return v;
}

void or_map(int w, int kind, int op, double p, const void* in, void* out, int64_t n) {
  if (w == 4) {
    const float* a = (const float*)in;
    float* b = (float*)out;
    for (int64_t i = 0; i < n; ++i) b[i] = map_f32(kind, op, (float)p, a[i]);
  } else {
    const double* a = (const double*)in;
    double* b = (double*)out;
    for (int64_t i = 0; i < n; ++i) b[i] = map_f64(kind, op, p, a[i]);
  }
}

void or_map_dia(int w, int op, double p, const int32_t* offset, const void* in, void* out,
                int32_t nd, int32_t stride, int32_t N) {
  for (int32_t d = 0; d < nd; ++d) {
    int32_t lo, hi;
    dia_range(offset[d], N, &lo, &hi);
    int64_t base = (int64_t)d * stride - (offset[d] < 0 ? (int64_t)(N - stride) : 0);
    if (hi > lo) or_map(w, 1, op, p, (const char*)in + (size_t)w * (base + lo),
                        (char*)out + (size_t)w * (base + lo), hi - lo);
  }
}

/* ======================= Matrix Market input ======================= */

/* The i-th field of a line split at single spaces (JavaScript split(" ")),
 * copied into buf; empty when absent. */
static void mm_field(const char* line, int64_t n, int idx, char* buf, int cap) {
  int k = 0;
  int64_t i = 0;
  while (k < idx && i < n) {
    if (line[i] == ' ') ++k;
    ++i;
  }
  int m = 0;
  if (k == idx)
    while (i < n && line[i] != ' ' && m < cap - 1) buf[m++] = line[i++];
  buf[m] = 0;
}

/* JavaScript Number() of a decimal field (the test inputs are plain
 * decimal numbers, for which strtod is the same correctly rounded parse). */
static double mm_number(const char* line, int64_t n, int idx) {
  char buf[128];
  mm_field(line, n, idx, buf, (int)sizeof(buf));
  return strtod(buf, NULL);
}

/* read_MM_header (:1889-1911) + read_matrix_MM_files (:1956-1981) with
 * calculate_actual_nnz (:1914-1954). */
int or_mm_read(const char* text, int64_t len, int64_t* nrows, int64_t* ncols, int64_t* nentries,
               int32_t* field, int32_t* symmetric, int32_t* row, int32_t* col, double* val,
               int64_t* nnz) {
  /* lines: up to the last '\n' (load_file keeps the text after it for the
   * next slice, and the last slice's remainder is dropped) */
  int64_t end = len;
  while (end > 0 && text[end - 1] != '\n') --end;
  int64_t pos = 0;
  /* first line: field and symmetry */
  int64_t e0 = pos;
  while (e0 < end && text[e0] != '\n') ++e0;
  char f[64], sy[64];
  mm_field(text, e0, 3, f, sizeof f);
  mm_field(text, e0, 4, sy, sizeof sy);
  *field = !strcmp(f, "real") ? 0 : !strcmp(f, "integer") ? 1 : !strcmp(f, "pattern") ? 2
           : !strcmp(f, "complex") ? 3 : -1;
  *symmetric = !strcmp(sy, "symmetric");
  /* skip comment lines (the first line starts with '%' too) */
  while (pos < end && text[pos] == '%') {
    while (pos < end && text[pos] != '\n') ++pos;
    ++pos;
  }
  int64_t le = pos;
  while (le < end && text[le] != '\n') ++le;
  *nrows = (int64_t)mm_number(text + pos, le - pos, 0);
  *ncols = (int64_t)mm_number(text + pos, le - pos, 1);
  *nentries = (int64_t)mm_number(text + pos, le - pos, 2);
  pos = le + 1;
  if (*nentries > ((int64_t)1 << 27)) return -1;
  if (!row) return 0;
  int64_t count = 0, j = 0;
  const int pattern = *field == 2, sym = *symmetric;
  while (pos < end) {
    le = pos;
    while (le < end && text[le] != '\n') ++le;
    const char* ln = text + pos;
    const int64_t n = le - pos;
    const int32_t r = (int32_t)mm_number(ln, n, 0), c = (int32_t)mm_number(ln, n, 1);
    if (j < *nentries) {
      row[j] = r;
      col[j] = c;
    }
    if (sym) {
      if (!pattern) {
        const double v = mm_number(ln, n, 2);
        if (j < *nentries) val[j] = v;
        if (v < 0 || v > 0) count += (r == c) ? 1 : 2;
      } else {
        count += (r == c) ? 1 : 2;
      }
    } else if (!pattern) {
      const double v = mm_number(ln, n, 2);
      if (j < *nentries) val[j] = v;
      if (v < 0 || v > 0) count++;
    }
    j++;
    pos = le + 1;
  }
  if (count == 0) count = *nentries;
  *nnz = count;
  if (count > ((int64_t)1 << 28)) return -1;
  return 0;
}

static void mm_put(int w, void* out_val, int64_t i, double v) {
  if (w == 4) ((float*)out_val)[i] = (float)v;
  else ((double*)out_val)[i] = v;
}

int64_t or_mm_coo(int w, int lower, int32_t field, int32_t symmetric, int64_t nrows,
                  int64_t nentries, int64_t nnz, const int32_t* row, const int32_t* col,
                  const double* val, int32_t* out_row, int32_t* out_col, void* out_val) {
  const int pattern = field == 2;
  int64_t i = 0;
  if (!lower) {
    /* create_COO_from_MM :2103-2172 */
    for (int64_t n = 0; n < nentries; ++n) {
      const double v = pattern ? 1.0 : val[n];
      if (!pattern && !(v < 0 || v > 0)) continue;
      out_row[i] = row[n] - 1;
      out_col[i] = col[n] - 1;
      mm_put(w, out_val, i, v);
      if (symmetric && row[n] != col[n]) {
        out_row[i + 1] = col[n] - 1;
        out_col[i + 1] = row[n] - 1;
        mm_put(w, out_val, i + 1, v);
        i += 2;
      } else {
        i += 1;
      }
    }
  } else {
    /* create_LCOO_from_MM :1983-2099: strictly lower part (mirrored upper
     * entries when symmetric), then the unit diagonal */
    for (int64_t n = 0; n < nentries; ++n) {
      const double v = pattern ? 1.0 : val[n];
      if (!pattern && !(v < 0 || v > 0)) continue;
      if (row[n] > col[n]) {
        out_row[i] = row[n] - 1;
        out_col[i] = col[n] - 1;
      } else if (symmetric && row[n] < col[n]) {
        out_row[i] = col[n] - 1;
        out_col[i] = row[n] - 1;
      } else {
        continue;
      }
      mm_put(w, out_val, i, v);
      i++;
    }
    for (int64_t n = 0; n < nrows; ++n) {
      out_row[i] = (int32_t)n;
      out_col[i] = (int32_t)n;
      mm_put(w, out_val, i, 1.0);
      i++;
    }
    nnz = i;
  }
  if (nnz > 0) or_quick_sort_coo(w, out_row, out_col, out_val, 0, nnz - 1);
  return nnz;
}

/* ======================= COO reductions ======================= */

#define OR_REDUCE(T, SFX)                                                                      \
  static void diag_##SFX(int32_t k, const int32_t* row, const int32_t* col, const T* val,     \
                         T* diag, int32_t N, int64_t nnz) {                                    \
    int32_t start = k < 0 ? -k : 0, end = k < 0 ? N : N - k;                                  \
    int64_t i = 0;                                                                             \
    /* $init: bring the pointer to the first row >= start */                                   \
    while (start > row[i]) {                                                                   \
      if (++i == nnz) return;                                                                  \
    }                                                                                          \
    for (;;) { /* $diag_loop */                                                                \
      while (row[i] == start) { /* $row_loop */                                                \
        if (col[i] - row[i] != k) {                                                            \
          if (++i == nnz) return;                                                              \
          continue;                                                                            \
        }                                                                                      \
        *diag = val[i]; /* found: skip the rest of the row */                                  \
        while (row[i] == start) {                                                              \
          if (++i == nnz) return;                                                              \
        }                                                                                      \
      }                                                                                        \
      diag++;                                                                                  \
      if (++start == end) return;                                                              \
    }                                                                                          \
  }                                                                                            \
  static void min_##SFX(int32_t axis, const int32_t* row, const T* val, T* out, int32_t N,     \
                        int64_t nnz) {                                                         \
    int64_t j = 0;                                                                             \
    T temp = 0;                                                                                \
    if (axis != 1) return;                                                                     \
    for (int32_t i = 0;;) { /* $min_loop_1 */                                                  \
      int32_t n = 0;                                                                           \
      if (row[j] == i) {                                                                       \
        temp = val[j];                                                                         \
        j++;                                                                                   \
        n++;                                                                                   \
        if (j == nnz) return;                                                                  \
      }                                                                                        \
      while (row[j] == i) { /* $row_loop_1 */                                                  \
        if (temp > val[j]) temp = val[j];                                                      \
        j++;                                                                                   \
        n++;                                                                                   \
        if (j == nnz) {                                                                        \
          if (n < N && 0 < temp) temp = 0;                                                     \
          *out = temp;                                                                         \
          return;                                                                              \
        }                                                                                      \
      }                                                                                        \
      if (n < N && 0 < temp) temp = 0;                                                         \
      *out = temp;                                                                             \
      out++;                                                                                   \
      if (++i == N) return;                                                                    \
    }                                                                                          \
  }                                                                                            \
  static void sumr_##SFX(int32_t axis, const int32_t* row, const T* val, T* out, int32_t N,    \
                         int64_t nnz) {                                                        \
    if (axis != 1) return;                                                                     \
    for (int32_t i = 0; i < N; ++i) out[i] = 0;                                                \
    for (int64_t e = 0; e < nnz; ++e) out[row[e]] = out[row[e]] + val[e];                      \
  }

OR_REDUCE(float, f32)
OR_REDUCE(double, f64)

void or_diagonal_coo(int w, int32_t k, const int32_t* row, const int32_t* col, const void* val,
                     void* diag, int32_t N, int64_t nnz) {
  if (nnz <= 0 || (int64_t)N - (k < 0 ? -(int64_t)k : k) <= 0) return;
  if (w == 4) diag_f32(k, row, col, (const float*)val, (float*)diag, N, nnz);
  else diag_f64(k, row, col, (const double*)val, (double*)diag, N, nnz);
}

void or_min_coo(int w, int32_t axis, const int32_t* row, const void* val, void* out, int32_t N,
                int64_t nnz) {
  if (N <= 0) return;
  if (nnz <= 0) { /* every row empty: the accumulator stays 0 */
    return;
  }
  if (w == 4) min_f32(axis, row, (const float*)val, (float*)out, N, nnz);
  else min_f64(axis, row, (const double*)val, (double*)out, N, nnz);
}

void or_sum_coo_rows(int w, int32_t axis, const int32_t* row, const void* val, void* out,
                     int32_t N, int64_t nnz) {
  if (w == 4) sumr_f32(axis, row, (const float*)val, (float*)out, N, nnz);
  else sumr_f64(axis, row, (const double*)val, (double*)out, N, nnz);
}

/* ======================= row reordering ======================= */

void or_sort_rows_by_nnz(int w, const int32_t* row_ptr, const int32_t* col, const void* val,
                         int32_t N, int32_t* nrow_ptr, int32_t* ncol, void* nval,
                         int32_t* nnz_per_row, int32_t* permutation, int32_t* small_rows) {
  int32_t* freq = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
  int32_t* start = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
  for (int32_t i = 0; i < N; ++i) {
    nnz_per_row[i] = row_ptr[i + 1] - row_ptr[i];
    freq[nnz_per_row[i]]++;
  }
  start[0] = 0;
  for (int32_t i = 1; i <= N; ++i) start[i] = start[i - 1] + freq[i - 1];
  small_rows[0] = N > 0 ? freq[0] : 0;
  for (int q = 1; q < 4; ++q) small_rows[q] = small_rows[q - 1] + (q <= N ? freq[q] : 0);
  for (int32_t i = 0; i < N; ++i) permutation[start[nnz_per_row[i]]++] = i;
  int64_t j = 0;
  nrow_ptr[0] = 0;
  for (int32_t i = 0; i < N; ++i) {
    int64_t k = row_ptr[permutation[i]];
    int32_t t = nnz_per_row[permutation[i]];
    nrow_ptr[i + 1] = nrow_ptr[i] + t;
    for (; t != 0; --t, ++j, ++k) {
      ncol[j] = col[k];
      memcpy((char*)nval + j * w, (const char*)val + k * w, (size_t)w);
    }
  }
  /* the reference's nnz_per_row array holds the lengths in the original
   * row order; the reordered matrix's lengths follow the permutation */
  for (int32_t i = 0; i < N; ++i) nnz_per_row[i] = nrow_ptr[i + 1] - nrow_ptr[i];
  free(freq);
  free(start);
}

void or_unpermute_rows(int w, const int32_t* permutation, const void* in, void* out, int32_t N) {
  for (int32_t i = 0; i < N; ++i)
    memcpy((char*)out + (size_t)permutation[i] * w, (const char*)in + (size_t)i * w, (size_t)w);
}

double or_csr_locality_index(const int32_t* row_ptr, const int32_t* col, int32_t N, int64_t nnz) {
  const int64_t lines = N / 16 + 1;
  int32_t* last_used = (int32_t*)malloc(sizeof(int32_t) * (size_t)lines);
  int32_t* reuse = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
  for (int64_t l = 0; l < lines; ++l) last_used[l] = -1;
  for (int32_t i = 0; i < N; ++i)
    for (int32_t j = row_ptr[i]; j < row_ptr[i + 1]; ++j) {
      const int64_t l = col[j] / 16;
      if (last_used[l] == -1) {
        last_used[l] = i;
        continue;
      }
      const int32_t d = i - last_used[l];
      if (d <= i) reuse[d]++;
      last_used[l] = i;
    }
  double sum = 0;
  for (int32_t d = 0; d < 16 && d <= N; ++d) sum += reuse[d];
  free(last_used);
  free(reuse);
  return (sum * 100) / (double)nnz;
}

/* ======================= CSC SpTS ======================= */

#define OR_SPTS_CSC(T, SFX)                                                                   \
  static void spts_csc_##SFX(const int32_t* cp, const int32_t* row, const T* val, const T* x, \
                             T* y, int32_t N) {                                               \
    for (int32_t j = 0; j < N; ++j) y[j] = x[j];                                              \
    for (int32_t j = 0; j < N; ++j) {                                                         \
      const int32_t s = cp[j], e = cp[j + 1];                                                 \
      y[j] = y[j] / val[s];                                                                   \
      for (int32_t q = s + 1; q < e; ++q) y[row[q]] = y[row[q]] - val[q] * y[j];              \
    }                                                                                         \
  }
OR_SPTS_CSC(float, f32)
OR_SPTS_CSC(double, f64)

void or_spts_csc(int w, const int32_t* cp, const int32_t* row, const void* val, const void* x,
                 void* y, int32_t N) {
  if (N <= 0) return;
  if (w == 4) spts_csc_f32(cp, row, (const float*)val, (const float*)x, (float*)y, N);
  else spts_csc_f64(cp, row, (const double*)val, (const double*)x, (double*)y, N);
}

/* ======================= nearest-neighbour row reordering ======================= */

/* assign_w_min_elems: src/parallel/src/sparse32.js:2271-2318.  The list
 * holds float32 values in the FP32 build (a Float32Array, :2444) and doubles
 * in the FP64 build (a Float64Array, src/parallel/src/sparse64.js:1593);
 * jac is kept in doubles here and `r32` rounds each stored value to float32
 * for the FP32 build.  -1 = empty; values compare as doubles with the new
 * candidate's double value.  An equal value goes after the existing ones; a
 * middle insertion into a partly filled list shifts from the last filled
 * slot, which drops that slot's entry (the list does not grow). */
static double nn_store(double v, int r32) { return r32 ? (double)(float)v : v; }

static void nn_assign(double* jac, int32_t* nidx, int32_t next, double v, int w, int r32) {
  int i = 0;
  while (i < w && jac[i] >= 0 && jac[i] >= v) i++;
  if (i == w) return;
  if (jac[i] == -1.0) {
    jac[i] = nn_store(v, r32);
    nidx[i] = next;
    return;
  }
  int j = w - 1;
  while (jac[j] == -1.0) j--;
  while (j != i) {
    jac[j] = jac[j - 1];
    nidx[j] = nidx[j - 1];
    j--;
  }
  jac[i] = nn_store(v, r32);
  nidx[i] = next;
}

/* find_next_row: src/parallel/src/sparse32.js:2321-2394.  A row that has
 * just joined the window (visited 3) gets its list: the w unvisited rows of
 * [start, end) with the highest Jaccard similarity of 16-column cache lines
 * (shared line runs / (its runs + their runs - shared runs)).  Returns the
 * first unvisited row of the row's list (N if none) and its value. */
static int32_t nn_find_next(int32_t index, int32_t* visited, const int32_t* nlines, double* jac,
                            int32_t* nidx, int32_t* last_used, const int32_t* row_ptr,
                            const int32_t* col, int32_t N, int w, int32_t start, int32_t end,
                            double* maxv, int r32) {
  if (visited[index] == 3) {
    visited[index] = 1;
    for (int i = 0; i < w; ++i) {
      jac[i] = -1.0;
      nidx[i] = N;
    }
    for (int32_t j = row_ptr[index]; j < row_ptr[index + 1]; ++j) last_used[col[j] / 16] = index;
    for (int32_t i = start; i < end; ++i) {
      if (visited[i] != 0) continue;
      int32_t j = row_ptr[i], alines = 0;
      while (j < row_ptr[i + 1]) {
        if (last_used[col[j] / 16] == index) alines++;
        j++;
        while (j < row_ptr[i + 1] && col[j - 1] / 16 == col[j] / 16) j++;
      }
      const int32_t dissim = nlines[index] + nlines[i] - alines;
      nn_assign(jac, nidx, i, (double)alines / (double)dissim, w, r32);
    }
  }
  for (int i = 0; i < w; ++i) {
    if (jac[i] >= 0 && visited[nidx[i]] == 0) {
      *maxv = jac[i];
      return nidx[i];
    }
  }
  *maxv = 0.0;
  return N;
}

/* reorder_subset: src/parallel/src/sparse32.js:2415-2483.  A greedy walk
 * from row `start`: each visited row joins a ring window of the last w rows;
 * the next row is the best first candidate over the window's lists (a later
 * window slot wins a tie), until no candidate is left. */
static void nn_subset(const int32_t* row_ptr, const int32_t* col, int32_t N, int32_t start,
                      int32_t end, const int32_t* nlines, int32_t* visited, int32_t* perm, int w,
                      int r32) {
  int32_t* win = (int32_t*)calloc((size_t)w, sizeof(int32_t));
  const int32_t nl = N / 16 + 1;
  int32_t* last_used = (int32_t*)malloc(sizeof(int32_t) * (size_t)nl);
  for (int32_t i = 0; i < nl; ++i) last_used[i] = -1;
  double* jac = (double*)calloc((size_t)w * w, sizeof(double));
  int32_t* nidx = (int32_t*)calloc((size_t)w * w, sizeof(int32_t));
  int32_t index = start, pos = start;
  int nnb = 0, count = 0;
  while (index != N) {
    visited[index] = 3;
    win[count++] = index;
    if (nnb < w) nnb++;
    if (count == w) count = 0;
    perm[pos++] = index;
    int32_t next = N;
    double mx = 0.0;
    for (int i = 0; i < nnb; ++i) {
      double v = 0.0;
      const int32_t c = nn_find_next(win[i], visited, nlines, jac + (size_t)i * w,
                                     nidx + (size_t)i * w, last_used, row_ptr, col, N, w, start,
                                     end, &v, r32);
      if (mx <= v && c != N) {
        mx = v;
        next = c;
      }
    }
    index = next;
  }
  free(win);
  free(last_used);
  free(jac);
  free(nidx);
}

/* reorder_NN: src/parallel/src/sparse32.js:2501-2622.  Empty rows are
 * skipped (visited 2); each row's number of line runs is counted; from the
 * first non-empty row on, consecutive position ranges sized by the row-length
 * histogram (lengths 1, 2, ..., in chunks of at most 1024 rows) are walked
 * independently.  With rows sorted by length (the reference calls it on the
 * output of sort_rows_by_nnz) each range holds rows of one length.  Outputs
 * the walk order `walk` (positions outside every range keep their index),
 * the new CSR (row i = input row walk[i]) and the permutation composed with
 * perm_in (new row i = original row perm_in[walk[i]]; perm_in NULL = the
 * identity).  The reference's new row_ptr view has length nrows + 1 with
 * nrows undefined, so it writes no row pointers; here they are written. */
void or_reorder_nn_ex(int w_bytes, int list_bytes, const int32_t* row_ptr, const int32_t* col,
                      const void* val, int32_t N, int w, const int32_t* perm_in, int32_t* walk,
                      int32_t* perm_out, int32_t* new_row, int32_t* new_col, void* new_val) {
  const int r32 = list_bytes == 4;
  int32_t* visited = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
  int32_t* nlines = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
  int32_t* freq = (int32_t*)calloc((size_t)N + 1, sizeof(int32_t));
  for (int32_t i = 0; i < N; ++i) {
    walk[i] = i;
    const int32_t len = row_ptr[i + 1] - row_ptr[i];
    freq[len]++;
    if (len == 0) visited[i] = 2;
  }
  for (int32_t i = 0; i < N; ++i) {
    if (visited[i] != 0) continue;
    int32_t j = row_ptr[i];
    while (j < row_ptr[i + 1]) {
      nlines[i]++;
      j++;
      while (j < row_ptr[i + 1] && col[j - 1] / 16 == col[j] / 16) j++;
    }
  }
  int32_t start = 0;
  while (start < N && visited[start] != 0) start++;
  if (start < N) {
    const int32_t B = 1024;
    for (int32_t len = 1; len < N + 1; ++len) {
      while (freq[len] >= B) {
        const int32_t end = start + B;
        freq[len] -= B;
        nn_subset(row_ptr, col, N, start, end, nlines, visited, walk, w, r32);
        start = end;
      }
      if (freq[len] > 0) {
        const int32_t end = start + freq[len];
        freq[len] = 0;
        nn_subset(row_ptr, col, N, start, end, nlines, visited, walk, w, r32);
        start = end;
      }
    }
  }
  int64_t o = 0;
  new_row[0] = 0;
  for (int32_t i = 0; i < N; ++i) {
    const int32_t s = walk[i];
    for (int32_t k = row_ptr[s]; k < row_ptr[s + 1]; ++k, ++o) {
      new_col[o] = col[k];
      copy_elem(new_val, o, val, k, w_bytes);
    }
    new_row[i + 1] = (int32_t)o;
    perm_out[i] = perm_in ? perm_in[s] : s;
  }
  free(visited);
  free(nlines);
  free(freq);
}

/* The FP32 build's list (float32 values) whatever the value width: the rule
 * the device follows for both precisions. */
void or_reorder_nn(int w_bytes, const int32_t* row_ptr, const int32_t* col, const void* val,
                   int32_t N, int w, const int32_t* perm_in, int32_t* walk, int32_t* perm_out,
                   int32_t* new_row, int32_t* new_col, void* new_val) {
  or_reorder_nn_ex(w_bytes, 4, row_ptr, col, val, N, w, perm_in, walk, perm_out, new_row, new_col,
                   new_val);
}
