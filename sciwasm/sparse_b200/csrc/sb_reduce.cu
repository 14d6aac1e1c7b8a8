// sb_reduce.cu -- reductions over a row-sorted COO matrix: diagonal_coo,
// min_coo and sum_coo (src/sequential/src/sparse_opt_32.wat:1707-1946;
// the JS methods A.diagonal(offset) and A.min(axis),
// src/sequential/src/sparse32.js:314-328).
//
// The reference walks the entries with one pointer, so it needs rows in
// non-decreasing order (its COO objects are quick-sorted by (row, col) after
// reading).  Here the rows are checked to be sorted, row pointers are built
// from them, and one thread per row folds that row's entries in storage
// order, which reproduces the reference's arithmetic exactly:
//  * diagonal_coo(k): slot i = the first entry of row start+i whose column is
//    row + k, else 0 (rows [max(0,-k), min(N, N-k))).
//  * min_coo(1): the fold t = first; t = (t > v) ? v : t, then 0 when the row
//    has fewer than N entries and 0 < t.  The reference's walk also makes an
//    empty row repeat the previous stored minimum when that is <= 0 (its
//    accumulator is not reset), leaves the last entry's row at 0 when it
//    holds a single entry (it returns before storing), and leaves every row
//    after the last entry's row at 0; all three are reproduced.
//  * sum_coo(1): the sum of each row in storage order.  The reference's
//    export increments its row counter for every entry it adds (:1800-1845),
//    so its output is not a row sum; this is the sum its loop structure and
//    min_coo's describe.  axis != 1 leaves the output at 0 for both, as in
//    the reference.
#include <algorithm>

#include "sb_common.cuh"
#include "sb_prims.cuh"

namespace sb {
namespace {

constexpr int kT = 256;

unsigned grid_n(long long n) {
  const long long g = (n + kT - 1) / kT;
  return (unsigned)std::max(1LL, std::min(g, 0x7fffffffLL));
}

__global__ void rows_sorted_check(const int* __restrict__ row, long long nnz, int N,
                                  int* __restrict__ flag) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
       i += (long long)gridDim.x * blockDim.x) {
    const int r = row[i];
    if (r < 0 || r >= N || (i + 1 < nnz && r > row[i + 1])) flag[0] = 1;
  }
}

template <typename T>
__global__ void diag_rows(const int* __restrict__ rp, const int* __restrict__ col,
                          const T* __restrict__ val, int k, int start, int count,
                          T* __restrict__ diag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int r = start + i;
  T d = 0;
  for (int e = rp[r]; e < rp[r + 1]; ++e)
    if (col[e] - r == k) {
      d = val[e];
      break;
    }
  diag[i] = d;
}

template <typename T>
__global__ void sum_rows(const int* __restrict__ rp, const T* __restrict__ val, int N,
                         T* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  T t = 0;
  for (int e = rp[i]; e < rp[i + 1]; ++e) t = t + val[e];
  out[i] = t;
}

// Stored minimum of each non-empty row (fold, then the implicit-zero rule);
// nonempty[i] = 1 for rows with entries.
template <typename T>
__global__ void min_rows(const int* __restrict__ rp, const T* __restrict__ val, int N,
                         T* __restrict__ stored, int* __restrict__ nonempty) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int s = rp[i], e = rp[i + 1];
  if (e == s) {
    nonempty[i] = 0;
    stored[i] = 0;
    return;
  }
  T t = val[s];
  for (int j = s + 1; j < e; ++j) {
    const T v = val[j];
    if (t > v) t = v;
  }
  if (e - s < N && (T)0 < t) t = 0;
  stored[i] = t;
  nonempty[i] = 1;
}

__global__ void compact_rows(const int* __restrict__ nonempty, const int* __restrict__ rank,
                             int N, int* __restrict__ idx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < N && nonempty[i]) idx[rank[i]] = i;
}

template <typename T>
__global__ void min_finish(const int* __restrict__ rp, const int* __restrict__ row, long long nnz,
                           const T* __restrict__ stored, const int* __restrict__ nonempty,
                           const int* __restrict__ rank, const int* __restrict__ idx, int N,
                           T* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int last = nnz > 0 ? row[nnz - 1] : -1;
  T v = 0;
  if (i <= last) {
    if (nonempty[i]) {
      v = (i == last && rp[i + 1] - rp[i] == 1) ? (T)0 : stored[i];
    } else if (rank[i] > 0) {
      const T p = stored[idx[rank[i] - 1]];  // the carried accumulator
      v = ((T)0 < p) ? (T)0 : p;
    }
  }
  out[i] = v;
}

// Row pointers of a row-sorted COO (SB_EINVAL when the rows are not sorted
// or out of range).  rp holds N + 1 entries.
int sorted_row_ptr(const int* row, long long nnz, int N, int* rp, const char* fn,
                   cudaStream_t st) {
  int* flag = nullptr;
  int r = scratch_alloc((void**)&flag, sizeof(int), st);
  if (r) return r;
  SB_CHECK_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), st));
  if (nnz > 0) {
    rows_sorted_check<<<std::min(grid_n(nnz), 4096u), kT, 0, st>>>(row, nnz, N, flag);
    SB_CHECK_LAUNCH("rows_sorted_check");
  }
  int h = 0;
  SB_CHECK_CUDA(cudaMemcpyAsync(&h, flag, sizeof(int), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  scratch_free(flag, st);
  if (h) {
    set_error("%s: rows must be sorted (non-decreasing) and in [0, N)", fn);
    return SB_EINVAL;
  }
  prim::row_ptr_from_sorted<<<grid_n(nnz + 1 > N + 1 ? nnz + 1 : N + 1), kT, 0, st>>>(row, nnz,
                                                                                    N, rp);
  SB_CHECK_LAUNCH("row_ptr_from_sorted");
  return SB_OK;
}

template <typename T>
int diagonal_impl(int k, const int* row, const int* col, const T* val, T* diag, int N,
                  long long nnz, cudaStream_t st) {
  const int start = k < 0 ? -k : 0;
  const int end = k < 0 ? N : N - k;
  const int count = end - start;
  int* rp = nullptr;
  int r = scratch_alloc((void**)&rp, sizeof(int) * ((size_t)N + 1), st);
  if (r) return r;
  if (!(r = sorted_row_ptr(row, nnz, N, rp, "sb_diagonal_coo", st))) {
    diag_rows<T><<<grid_n(count), kT, 0, st>>>(rp, col, val, k, start, count, diag);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "diag_rows");
  }
  scratch_free(rp, st);
  return r;
}

template <typename T>
int reduce_impl(bool is_min, const int* row, const T* val, T* out, int N, long long nnz,
                cudaStream_t st) {
  int* rp = nullptr;
  const size_t ints = (size_t)N + 1 + (is_min ? 3 * (size_t)N + 1 : 0);
  void* mem = nullptr;
  int r = scratch_alloc(&mem, sizeof(int) * ints + (is_min ? sizeof(T) * (size_t)N : 0), st);
  if (r) return r;
  rp = (int*)mem;
  if (!(r = sorted_row_ptr(row, nnz, N, rp, is_min ? "sb_min_coo" : "sb_sum_coo", st))) {
    if (!is_min) {
      sum_rows<T><<<grid_n(N), kT, 0, st>>>(rp, val, N, out);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) r = cuda_status(e, "sum_rows");
    } else {
      int* nonempty = rp + N + 1;
      int* rank = nonempty + N;
      int* idx = rank + N + 1;
      T* stored = (T*)(rp + ints);
      min_rows<T><<<grid_n(N), kT, 0, st>>>(rp, val, N, stored, nonempty);
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) r = cuda_status(e, "min_rows");
      if (!r) r = prim::exclusive_scan(nonempty, rank, N, st);
      if (!r) {
        compact_rows<<<grid_n(N), kT, 0, st>>>(nonempty, rank, N, idx);
        e = cudaGetLastError();
        if (e != cudaSuccess) r = cuda_status(e, "compact_rows");
      }
      if (!r) {
        min_finish<T><<<grid_n(N), kT, 0, st>>>(rp, row, nnz, stored, nonempty, rank, idx, N,
                                                out);
        e = cudaGetLastError();
        if (e != cudaSuccess) r = cuda_status(e, "min_finish");
      }
    }
  }
  scratch_free(mem, st);
  return r;
}

int check(int dtype, int N, long long nnz, const char* fn) {
  if (dtype != SB_F32 && dtype != SB_F64) {
    set_error("%s: dtype must be F32 or F64", fn);
    return SB_EINVAL;
  }
  if (N < 0 || nnz < 0 || nnz > 0x7fffffffLL) {
    set_error("%s: bad size", fn);
    return SB_EINVAL;
  }
  return ensure_device();
}

}  // namespace
}  // namespace sb

using namespace sb;

extern "C" {

int sb_diagonal_coo(int dtype, int32_t k, const int32_t* row, const int32_t* col,
                    const void* val, void* diag, int32_t N, int64_t nnz, void* stream) {
  SB_TRACE("sb_diagonal_coo");
  int r = check(dtype, N, nnz, "sb_diagonal_coo");
  if (r) return r;
  if ((long long)N - std::abs((long long)k) <= 0) {  // the reference returns no vector
    set_error("sb_diagonal_coo: |offset| must be below N");
    return SB_EINVAL;
  }
  SB_REQUIRE(diag && (nnz == 0 || (row && col && val)), "sb_diagonal_coo: null pointer");
  cudaStream_t st = as_stream(stream);
  if (dtype == SB_F32)
    return diagonal_impl<float>(k, row, col, (const float*)val, (float*)diag, N, nnz, st);
  return diagonal_impl<double>(k, row, col, (const double*)val, (double*)diag, N, nnz, st);
}

int sb_min_coo(int dtype, int32_t axis, const int32_t* row, const int32_t* col, const void* val,
               void* out, int32_t N, int64_t nnz, void* stream) {
  SB_TRACE("sb_min_coo");
  int r = check(dtype, N, nnz, "sb_min_coo");
  if (r) return r;
  SB_REQUIRE(out && (nnz == 0 || (row && col && val)), "sb_min_coo: null pointer");
  (void)col;
  if (axis != 1 || N == 0) return SB_OK;  // the reference only handles axis 1
  cudaStream_t st = as_stream(stream);
  if (dtype == SB_F32)
    return reduce_impl<float>(true, row, (const float*)val, (float*)out, N, nnz, st);
  return reduce_impl<double>(true, row, (const double*)val, (double*)out, N, nnz, st);
}

int sb_sum_coo(int dtype, int32_t axis, const int32_t* row, const int32_t* col, const void* val,
               void* out, int32_t N, int64_t nnz, void* stream) {
  SB_TRACE("sb_sum_coo");
  int r = check(dtype, N, nnz, "sb_sum_coo");
  if (r) return r;
  SB_REQUIRE(out && (nnz == 0 || (row && col && val)), "sb_sum_coo: null pointer");
  (void)col;
  if (axis != 1 || N == 0) return SB_OK;
  cudaStream_t st = as_stream(stream);
  if (dtype == SB_F32)
    return reduce_impl<float>(false, row, (const float*)val, (float*)out, N, nnz, st);
  return reduce_impl<double>(false, row, (const double*)val, (double*)out, N, nnz, st);
}

}  // extern "C"
