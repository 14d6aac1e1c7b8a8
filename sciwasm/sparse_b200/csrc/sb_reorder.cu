// sb_reorder.cu -- row reordering by row length and the CSR locality index
// (src/parallel/src/sparse32.js:2148-2269).
//
// sort_rows_by_nnz is a stable counting sort of the rows by their number of
// nonzeros followed by a CSR whose rows are gathered in that order (columns
// unchanged); here the rows are stably radix-sorted by length on the device,
// the new row_ptr is a scan of the permuted lengths and one thread per row
// copies its entries.  sort_y_rows_by_nnz scatters y back to the original
// row order.  calculate_csr_locality_index walks the entries in storage
// order and counts the accesses whose 16-column line was last touched fewer
// than 16 rows earlier; each access's previous touch of its line is its
// predecessor after a stable sort of the accesses by line, so the count is
// one sort, one comparison per access and a reduction.
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

__global__ void length_keys(const int* __restrict__ rp, int N, unsigned long long* __restrict__ k,
                            unsigned* __restrict__ v, int* __restrict__ len,
                            int* __restrict__ small) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int l = rp[i + 1] - rp[i];
  k[i] = (unsigned long long)(unsigned)l;
  v[i] = (unsigned)i;
  len[i] = l;
  if (l < 4) atomicAdd(small + l, 1);
}

__global__ void perm_lengths(const unsigned* __restrict__ sorted, const int* __restrict__ len,
                             int N, int* __restrict__ perm, int* __restrict__ plen) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int i = (int)sorted[p];
  perm[p] = i;
  plen[p] = len[i];
}

template <typename T>
__global__ void gather_rows(const int* __restrict__ rp, const int* __restrict__ col,
                            const T* __restrict__ val, const int* __restrict__ perm,
                            const int* __restrict__ nrp, int N, int* __restrict__ ncol,
                            T* __restrict__ nval) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int src = perm[p];
  int o = nrp[p];
  for (int j = rp[src]; j < rp[src + 1]; ++j, ++o) {
    ncol[o] = col[j];
    nval[o] = val[j];
  }
}

template <typename T>
__global__ void scatter_rows(const int* __restrict__ perm, const T* __restrict__ in, int N,
                             T* __restrict__ out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < N) out[perm[p]] = in[p];
}

__global__ void line_keys(const int* __restrict__ col, long long nnz,
                          unsigned long long* __restrict__ k, unsigned* __restrict__ v) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
       i += (long long)gridDim.x * blockDim.x) {
    k[i] = (unsigned long long)(unsigned)(col[i] / 16);
    v[i] = (unsigned)i;
  }
}

// Accesses (in line order) whose previous touch of the same line is fewer
// than 16 rows back.
__global__ void near_reuse(const unsigned long long* __restrict__ k,
                           const unsigned* __restrict__ pos, const int* __restrict__ row_of,
                           long long nnz, unsigned long long* __restrict__ count) {
  unsigned c = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nnz;
       i += (long long)gridDim.x * blockDim.x)
    if (i > 0 && k[i] == k[i - 1] && row_of[pos[i]] - row_of[pos[i - 1]] < 16) ++c;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, (unsigned long long)c);
}

template <typename T>
int sort_rows_impl(const int* rp, const int* col, const T* val, int N, long long nnz, int* nrp,
                   int* ncol, T* nval, int* nnz_per_row, int* perm, int32_t* small_rows,
                   cudaStream_t st) {
  const size_t kb = sizeof(unsigned long long) * (size_t)N, vb = sizeof(unsigned) * (size_t)N;
  void* mem = nullptr;
  int r = scratch_alloc(&mem, 2 * kb + 2 * vb + sizeof(int) * ((size_t)N + 4), st);
  if (r) return r;
  char* p = (char*)mem;
  prim::RadixBuffers b;
  b.k[0] = (unsigned long long*)p;
  b.k[1] = (unsigned long long*)(p + kb);
  b.v[0] = (unsigned*)(p + 2 * kb);
  b.v[1] = (unsigned*)(p + 2 * kb + vb);
  int* small = (int*)(p + 2 * kb + 2 * vb);
  int* len = small + 4;
  SB_CHECK_CUDA(cudaMemsetAsync(small, 0, 4 * sizeof(int), st));
  length_keys<<<grid_n(N), kT, 0, st>>>(rp, N, b.k[0], b.v[0], len, small);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) r = cuda_status(e, "length_keys");
  const int ranges[2] = {0, prim::bits_for(nnz)};
  int which = 0;
  if (!r) r = prim::radix_sort_ranges(b, N, ranges, 1, &which, st);
  if (!r) {
    perm_lengths<<<grid_n(N), kT, 0, st>>>(b.v[which], len, N, perm, nnz_per_row);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "perm_lengths");
  }
  if (!r) r = prim::exclusive_scan(nnz_per_row, nrp, N, st);
  if (!r) {
    const int nz = (int)nnz;
    e = cudaMemcpyAsync(nrp + N, &nz, sizeof(int), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) r = cuda_status(e, "row_ptr");
  }
  if (!r) {
    gather_rows<T><<<grid_n(N), kT, 0, st>>>(rp, col, val, perm, nrp, N, ncol, nval);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "gather_rows");
  }
  int h[4] = {0, 0, 0, 0};
  if (!r) {
    e = cudaMemcpyAsync(h, small, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "sb_sort_rows_by_nnz");
  }
  if (!r && small_rows) {  // cumulative: rows with at most 0, 1, 2, 3 nonzeros
    small_rows[0] = h[0];
    for (int q = 1; q < 4; ++q) small_rows[q] = small_rows[q - 1] + h[q];
  }
  scratch_free(mem, st);
  return r;
}

}  // namespace
}  // namespace sb

using namespace sb;

extern "C" {

int sb_sort_rows_by_nnz(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                        int32_t N, int64_t nnz, int32_t* out_row_ptr, int32_t* out_col,
                        void* out_val, int32_t* nnz_per_row, int32_t* permutation,
                        int32_t* small_rows, void* stream) {
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64, "sb_sort_rows_by_nnz: dtype must be F32 or F64");
  SB_REQUIRE(N >= 0 && nnz >= 0 && nnz <= 0x7fffffffLL, "sb_sort_rows_by_nnz: bad size");
  SB_REQUIRE(N == 0 || (row_ptr && out_row_ptr && nnz_per_row && permutation),
             "sb_sort_rows_by_nnz: null pointer");
  SB_REQUIRE(nnz == 0 || (col && val && out_col && out_val), "sb_sort_rows_by_nnz: null pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  if (N == 0) {
    if (small_rows) small_rows[0] = small_rows[1] = small_rows[2] = small_rows[3] = 0;
    if (out_row_ptr) SB_CHECK_CUDA(cudaMemsetAsync(out_row_ptr, 0, sizeof(int32_t), st));
    return SB_OK;
  }
  if (dtype == SB_F32)
    return sort_rows_impl<float>(row_ptr, col, (const float*)val, N, nnz, out_row_ptr, out_col,
                                 (float*)out_val, nnz_per_row, permutation, small_rows, st);
  return sort_rows_impl<double>(row_ptr, col, (const double*)val, N, nnz, out_row_ptr, out_col,
                                (double*)out_val, nnz_per_row, permutation, small_rows, st);
}

int sb_unpermute_rows(int dtype, const int32_t* permutation, const void* in, void* out,
                      int32_t N, void* stream) {
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64, "sb_unpermute_rows: dtype must be F32 or F64");
  SB_REQUIRE(N >= 0, "sb_unpermute_rows: bad size");
  if (N == 0) return SB_OK;
  SB_REQUIRE(permutation && in && out && in != out, "sb_unpermute_rows: bad pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  if (dtype == SB_F32)
    scatter_rows<float><<<grid_n(N), kT, 0, st>>>(permutation, (const float*)in, N, (float*)out);
  else
    scatter_rows<double><<<grid_n(N), kT, 0, st>>>(permutation, (const double*)in, N,
                                                   (double*)out);
  SB_CHECK_LAUNCH("scatter_rows");
  return SB_OK;
}

int sb_csr_locality_index(const int32_t* row_ptr, const int32_t* col, int32_t N, int64_t nnz,
                          double* index, void* stream) {
  SB_REQUIRE(index, "sb_csr_locality_index: null output");
  SB_REQUIRE(N >= 0 && nnz >= 0 && nnz <= 0x7fffffffLL, "sb_csr_locality_index: bad size");
  *index = 0.0;
  if (nnz == 0) {  // the reference's 0 * 100 / 0
    *index = __builtin_nan("");
    return SB_OK;
  }
  SB_REQUIRE(row_ptr && col, "sb_csr_locality_index: null pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  const size_t kb = sizeof(unsigned long long) * (size_t)nnz, vb = sizeof(unsigned) * (size_t)nnz;
  void* mem = nullptr;
  // [count (8 bytes)] [keys 2 x nnz u64] [positions 2 x nnz u32] [row of each entry]
  if ((r = scratch_alloc(&mem, 8 + 2 * kb + 2 * vb + sizeof(int) * (size_t)nnz, st))) return r;
  char* p = (char*)mem;
  unsigned long long* count = (unsigned long long*)p;
  p += 8;
  prim::RadixBuffers b;
  b.k[0] = (unsigned long long*)p;
  b.k[1] = (unsigned long long*)(p + kb);
  b.v[0] = (unsigned*)(p + 2 * kb);
  b.v[1] = (unsigned*)(p + 2 * kb + vb);
  int* row_of = (int*)(p + 2 * kb + 2 * vb);
  cudaError_t e = cudaSuccess;
  SB_CHECK_CUDA(cudaMemsetAsync(count, 0, sizeof(unsigned long long), st));
  prim::expand_rows<<<grid_n(N), kT, 0, st>>>(row_ptr, N, row_of);
  e = cudaGetLastError();
  if (e != cudaSuccess) r = cuda_status(e, "expand_rows");
  if (!r) {
    line_keys<<<std::min(grid_n(nnz), 4096u), kT, 0, st>>>(col, nnz, b.k[0], b.v[0]);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "line_keys");
  }
  const int ranges[2] = {0, prim::bits_for(N / 16)};
  int which = 0;
  if (!r) r = prim::radix_sort_ranges(b, nnz, ranges, 1, &which, st);
  if (!r) {
    near_reuse<<<std::min(grid_n(nnz), 4096u), kT, 0, st>>>(b.k[which], b.v[which], row_of, nnz,
                                                            count);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "near_reuse");
  }
  unsigned long long h = 0;
  if (!r) {
    e = cudaMemcpyAsync(&h, count, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "sb_csr_locality_index");
  }
  scratch_free(mem, st);
  if (!r) *index = ((double)h * 100.0) / (double)nnz;
  return r;
}

}  // extern "C"
