// sb_tune.cu -- SpMV format and kernel autotuner.
//
// No counterpart in the reference: its users pick a format by hand (coo_csr,
// csr_dia, csr_ell; src/sequential/src/sparse32.js:1436-1720) and its
// parallel harness times CSR variants per run (src/parallel/tests/main32.js).
// Here one call takes a CSR matrix and decides:
//   1. from its statistics (N, nnz, max row length nc, diagonal count nd):
//      which of DIA and ELL the reference's admission test allows
//      (w*N < 2^27 and w*N/nnz <= 5), and the compulsory bytes of one
//      y <- y + A x in every format;
//   2. in the statistics mode (SB_TUNE_MODEL): the admitted format with the
//      fewest bytes, and CSR kernel options from the row-length statistics;
//   3. in the timed mode (SB_TUNE_TIMED): every admitted format within twice
//      the CSR bytes (more cannot win on a bandwidth-bound device) timed with
//      CUDA events -- CSR with its kernel options from sb_csr_autotune
//      (kernel, lanes per row, unroll, grid), DIA and ELL built on the device
//      into scratch, COO with the row array expanded from row_ptr -- and the
//      fastest kept.
// The caller converts the matrix to the chosen format (and keeps it).
#include <algorithm>

#include "sb_common.cuh"
#include "sb_prims.cuh"

namespace sb {

static long long vec_bytes(long long N, int s) { return 3LL * N * s; }

static int time_calls(cudaStream_t st, int reps, float* ms, int (*call)(void*), void* ctx) {
  cudaEvent_t e0, e1;
  SB_CHECK_CUDA(cudaEventCreate(&e0));
  SB_CHECK_CUDA(cudaEventCreate(&e1));
  int r = call(ctx);  // warm-up
  if (!r) SB_CHECK_CUDA(cudaEventRecord(e0, st));
  for (int i = 0; i < reps && !r; ++i) r = call(ctx);
  if (!r) {
    cudaEventRecord(e1, st);
    cudaError_t e = cudaEventSynchronize(e1);
    if (e != cudaSuccess) r = cuda_status(e, "sb_spmv_autotune");
    else {
      cudaEventElapsedTime(ms, e0, e1);
      *ms /= reps;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return r;
}

// CSR kernel options from the row statistics alone: the row-block kernel
// with lanes per row from the mean length; rows whose longest is far above
// the mean (skewed, power-law-like) take one warp per 32-row block, so that
// blocks holding long rows do not hold back a fixed share of the others.
// (The block-stream kernel measured slower than the row-block kernel on every
// matrix tried, power law included, so the statistics never pick it.)
static sb_csr_opts csr_model_opts(int N, long long nnz, int max_row) {
  const double mean = N ? (double)nnz / N : 0.0;
  const int lanes = mean <= 6 ? 2 : mean <= 14 ? 4 : mean <= 28 ? 8 : 16;
  const int grid = (max_row > 0 && max_row > 8.0 * mean) ? 1 : 0;
  return sb_csr_opts{0, lanes, 4, grid};
}

struct TuneCtx {
  int dtype;
  const int32_t* a;  // offsets / indices / rows
  const int32_t* b;  // col (COO)
  const void* data;
  const void* x;
  void* y;
  int32_t N;
  int32_t w;
  int64_t nnz;
  void* stream;
};

static int call_dia(void* p) {
  TuneCtx* c = (TuneCtx*)p;
  return sb_spmv_dia(c->dtype, c->a, c->data, c->N, c->w, c->N, c->x, c->y, 1, c->stream);
}
static int call_ell(void* p) {
  TuneCtx* c = (TuneCtx*)p;
  return sb_spmv_ell(c->dtype, c->a, c->data, c->N, c->w, c->x, c->y, 1, c->stream);
}
static int call_coo(void* p) {
  TuneCtx* c = (TuneCtx*)p;
  return sb_spmv_coo_ex(c->dtype, c->a, c->b, c->data, c->x, c->y, c->N, c->nnz, 1,
                        SB_COO_ROWS_SORTED, c->stream);
}

}  // namespace sb

using namespace sb;

extern "C" {

int sb_spmv_autotune(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                     const void* x, int32_t N, int64_t nnz, int32_t mode, int32_t reps,
                     sb_spmv_choice* out, void* stream) {
  SB_TRACE("sb_spmv_autotune");
  SB_REQUIRE(out, "sb_spmv_autotune: null output");
  *out = sb_spmv_choice{};
  for (int k = 0; k < 4; ++k) out->ms[k] = -1.f;
  out->format = SB_FMT_CSR;
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64 || dtype == SB_BF16,
             "sb_spmv_autotune: bad dtype %d", dtype);
  SB_REQUIRE(mode == SB_TUNE_MODEL || mode == SB_TUNE_TIMED, "sb_spmv_autotune: bad mode %d",
             mode);
  SB_REQUIRE(N >= 0 && nnz >= 0 && nnz <= 0x7fffffffLL, "sb_spmv_autotune: bad size");
  int r = SB_OK;
  out->csr = csr_model_opts(N, nnz, 0);
  if (N == 0 || nnz == 0) return r;
  cudaStream_t st = as_stream(stream);
  const int s = dtype == SB_F64 ? 8 : (dtype == SB_F32 ? 4 : 2);
  const int sx = dtype == SB_F64 ? 8 : 4;  // BF16 values use f32 vectors
  int32_t nc = 0, nd = 0, stride = 0;
  if ((r = sb_num_cols(row_ptr, N, &nc, stream))) return r;
  if ((r = sb_num_diags(row_ptr, col, N, &nd, &stride, stream))) return r;
  out->ncols = nc;
  out->ndiags = nd;
  out->ell_admitted = sb_ell_admitted(nc, N, nnz);
  out->dia_admitted = sb_dia_admitted(nd, stride, nnz);
  out->csr = csr_model_opts(N, nnz, nc);
  const long long b_csr = nnz * (s + 4) + 4LL * (N + 1) + vec_bytes(N, sx);
  const long long b_dia = (long long)nd * N * s + 4LL * nd + vec_bytes(N, sx);
  const long long b_ell = (long long)nc * N * (s + 4) + vec_bytes(N, sx);
  const long long b_coo = nnz * (s + 8) + vec_bytes(N, sx);
  out->bytes[0] = b_csr;
  out->bytes[1] = b_dia;
  out->bytes[2] = b_ell;
  out->bytes[3] = b_coo;
  if (mode == SB_TUNE_MODEL) {
    // fewest compulsory bytes among the admitted formats; CSR on a tie (COO
    // never moves fewer bytes than CSR)
    long long best = b_csr;
    if (out->dia_admitted && b_dia < best) {
      best = b_dia;
      out->format = SB_FMT_DIA;
    }
    if (out->ell_admitted && b_ell < best) out->format = SB_FMT_ELL;
    return SB_OK;
  }
  r = sb_csr_autotune(dtype, row_ptr, col, val, x, N, nnz, reps, &out->csr, &out->ms[0], stream);
  // BF16 values have only the CSR single-call kernel
  if (r || dtype == SB_BF16) return r;
  if (reps <= 0) reps = 5;
  void* ywork = nullptr;
  if ((r = scratch_alloc(&ywork, (size_t)s * N, st))) return r;
  SB_CHECK_CUDA(cudaMemsetAsync(ywork, 0, (size_t)s * N, st));
  TuneCtx c{dtype, nullptr, nullptr, nullptr, x, ywork, N, 0, nnz, stream};
  if (out->dia_admitted && b_dia <= 2 * b_csr) {
    void* mem = nullptr;
    const size_t off_b = ((sizeof(int) * (size_t)nd + 255) / 256) * 256;
    if (!(r = scratch_alloc(&mem, off_b + (size_t)s * nd * N, st))) {
      int32_t* off = (int32_t*)mem;
      void* data = (char*)mem + off_b;
      r = sb_csr_dia(dtype, row_ptr, col, val, N, nnz, nd, N, off, data, stream);
      c.a = off;
      c.data = data;
      c.w = nd;
      if (!r) r = time_calls(st, reps, &out->ms[1], call_dia, &c);
      scratch_free(mem, st);
    }
  }
  if (!r && out->ell_admitted && b_ell <= 2 * b_csr) {
    void* mem = nullptr;
    const size_t ib = (((size_t)4 * nc * N + 255) / 256) * 256;
    if (!(r = scratch_alloc(&mem, ib + (size_t)s * nc * N, st))) {
      int32_t* ind = (int32_t*)mem;
      void* data = (char*)mem + ib;
      r = sb_csr_ell(dtype, row_ptr, col, val, N, nnz, nc, ind, data, stream);
      c.a = ind;
      c.data = data;
      c.w = nc;
      if (!r) r = time_calls(st, reps, &out->ms[2], call_ell, &c);
      scratch_free(mem, st);
    }
  }
  if (!r && b_coo <= 2 * b_csr) {
    int32_t* rows = nullptr;
    if (!(r = scratch_alloc((void**)&rows, sizeof(int32_t) * (size_t)nnz, st))) {
      prim::expand_rows<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(row_ptr, N, rows);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) r = cuda_status(e, "expand_rows");
      c.a = rows;
      c.b = col;
      c.data = val;
      if (!r) r = time_calls(st, reps, &out->ms[3], call_coo, &c);
      scratch_free(rows, st);
    }
  }
  scratch_free(ywork, st);
  if (r) return r;
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  int best = 0;
  for (int k = 1; k < 4; ++k)
    if (out->ms[k] >= 0.f && out->ms[k] < out->ms[best]) best = k;
  out->format = best;  // SB_FMT_CSR, SB_FMT_DIA, SB_FMT_ELL, SB_FMT_COO
  return SB_OK;
}

int sb_csr_coo(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val, int32_t N,
               int64_t nnz, int32_t* coo_row, int32_t* coo_col, void* coo_val, void* stream) {
  SB_TRACE("sb_csr_coo");
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64 || dtype == SB_BF16, "sb_csr_coo: bad dtype");
  SB_REQUIRE(N >= 0 && nnz >= 0, "sb_csr_coo: negative size");
  if (N == 0 || nnz == 0) return SB_OK;
  SB_REQUIRE(row_ptr && col && val && coo_row && coo_col && coo_val, "sb_csr_coo: null pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  prim::expand_rows<<<(unsigned)((N + 255) / 256), 256, 0, st>>>(row_ptr, N, coo_row);
  SB_CHECK_LAUNCH("expand_rows");
  SB_CHECK_CUDA(cudaMemcpyAsync(coo_col, col, sizeof(int32_t) * (size_t)nnz,
                                cudaMemcpyDeviceToDevice, st));
  SB_CHECK_CUDA(cudaMemcpyAsync(coo_val, val, dtype_size(dtype) * (size_t)nnz,
                                cudaMemcpyDeviceToDevice, st));
  return SB_OK;
}

}  // extern "C"
