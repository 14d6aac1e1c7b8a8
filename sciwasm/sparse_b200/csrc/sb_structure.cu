// sb_structure.cu -- eliminate_zeros and transpose for COO/CSR/DIA/ELL on the
// device, bit-exact with the reference's wasm kernels
// (src/sequential/src/sparse_opt_32.wat):
//   count_nonzeros_coo :500, copy_nonzeros_coo :523, copy_nonzeros_csr :548,
//   count/copy_nonzeros_dia :1948/:2041, count/copy_nonzeros_ell :5821/:5895,
//   transpose_csr :6348, transpose_dia :6479, count_transpose_cols_ell :6574,
//   transpose_ell :6634; COO transpose swaps the index arrays
//   (src/sequential/src/sparse32.js:1106-1115).
// The nonzero test everywhere is v > 0 || v < 0 (+0, -0 and NaN are zeros).
// Ordered compactions use an exclusive scan of the keep flags; orderings
// that the reference gets from sequential counting sorts use the stable
// radix sort with the original position as payload.
#include <algorithm>

#include "sb_common.cuh"
#include "sb_prims.cuh"

namespace sb {

constexpr int kTh = 256;

static unsigned g1(long long n) {
  long long g = (n + kTh - 1) / kTh;
  return (unsigned)std::max(1LL, std::min(g, 0x7fffffffLL));
}

template <typename T> __device__ __forceinline__ bool nz(T v) { return v > (T)0 || v < (T)0; }

template <typename T>
__global__ void count_nz(const T* __restrict__ v, long long n, unsigned long long* __restrict__ out) {
  unsigned long long c = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    c += nz(v[i]) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

template <typename T>
__global__ void nz_flags(const T* __restrict__ v, long long n, int* __restrict__ f) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) f[i] = nz(v[i]) ? 1 : 0;
  else if (i == n) f[i] = 0;
}

template <typename T>
__global__ void scatter_nz_coo(const int* __restrict__ row, const int* __restrict__ col,
                               const T* __restrict__ val, long long n, const int* __restrict__ pos,
                               int* __restrict__ orow, int* __restrict__ ocol, T* __restrict__ oval) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !nz(val[i])) return;
  const int p = pos[i];
  if (orow) orow[p] = row[i];
  ocol[p] = col[i];
  oval[p] = val[i];
}

__global__ void rowptr_through(const int* __restrict__ row_ptr, int N, const int* __restrict__ pos,
                               int* __restrict__ orow_ptr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i <= N) orow_ptr[i] = pos[row_ptr[i]];
}

// DIA: keep flags over the virtual (diagonal, row) grid d*N + n, in-band only.
template <typename T>
__global__ void dia_nz_flags(const int* __restrict__ offset, const T* __restrict__ data, int nd,
                             int stride, int N, int* __restrict__ f) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)nd * N;
  if (q > total) return;
  if (q == total) {
    f[q] = 0;
    return;
  }
  const int d = (int)(q / N), n = (int)(q - (long long)d * N);
  const int k = offset[d];
  const bool in = (unsigned)(n + k) < (unsigned)N;
  const long long idx = (long long)d * stride + n - (k < 0 ? (long long)(N - stride) : 0);
  f[q] = (in && nz(data[idx])) ? 1 : 0;
}

__global__ void dia_kept(const int* __restrict__ pos, int nd, int N, int* __restrict__ kept) {
  const int d = blockIdx.x * blockDim.x + threadIdx.x;
  if (d < nd) kept[d] = (pos[(long long)(d + 1) * N] - pos[(long long)d * N]) > 0 ? 1 : 0;
  else if (d == nd) kept[d] = 0;
}

template <typename T>
__global__ void dia_copy_nz(const int* __restrict__ offset, const T* __restrict__ data, int nd,
                            int stride, int N, const int* __restrict__ pos,
                            const int* __restrict__ slot, int* __restrict__ ooffset,
                            T* __restrict__ odata) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)nd * N) return;
  const int d = (int)(q / N), n = (int)(q - (long long)d * N);
  const int k = offset[d];
  const long long base = (long long)d * N;
  if (n == 0 && pos[base + N] > pos[base]) ooffset[slot[d]] = k;
  const bool in = (unsigned)(n + k) < (unsigned)N;
  if (!in) return;
  const long long idx = (long long)d * stride + n - (k < 0 ? (long long)(N - stride) : 0);
  if (!nz(data[idx])) return;
  const int lo = k < 0 ? -k : 0;
  const long long t = pos[q] - pos[base];
  odata[(long long)slot[d] * stride + lo + t] = data[idx];
}

// ELL: per-row nonzero counts; copy packs each row's nonzeros in slot order.
template <typename T>
__global__ void ell_row_counts(const T* __restrict__ data, int nc, int N, int* __restrict__ cnt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int c = 0;
  for (int k = 0; k < nc; ++k) c += nz(data[(long long)k * N + i]) ? 1 : 0;
  cnt[i] = c;
}

__global__ void max_sum(const int* __restrict__ a, int n, int* __restrict__ mx,
                        unsigned long long* __restrict__ sum) {
  int m = 0;
  unsigned long long s = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    m = max(m, a[i]);
    s += (unsigned)a[i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    s += __shfl_xor_sync(0xffffffffu, s, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(mx, m);
    if (sum && s) atomicAdd(sum, s);
  }
}

template <typename T>
__global__ void ell_copy_nz(const T* __restrict__ data, const int* __restrict__ idx, int nc, int N,
                            int onc, T* __restrict__ odata, int* __restrict__ oidx) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  int o = 0;
  for (int k = 0; k < nc; ++k) {
    const long long s = (long long)k * N + i;
    const T v = data[s];
    if (nz(v) && o < onc) {
      odata[(long long)o * N + i] = v;
      oidx[(long long)o * N + i] = idx[s];
      ++o;
    }
  }
  for (; o < onc; ++o) {
    odata[(long long)o * N + i] = (T)0;
    oidx[(long long)o * N + i] = 0;
  }
}

// transpose_csr: sort entries (storage order) stably by column.
__global__ void col_keys(const int* __restrict__ col, long long nnz,
                         unsigned long long* __restrict__ k, unsigned* __restrict__ v) {
  const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nnz) {
    k[j] = (unsigned long long)(unsigned)col[j];
    v[j] = (unsigned)j;
  }
}

template <typename T>
__global__ void transpose_gather(const unsigned long long* __restrict__ k,
                                 const unsigned* __restrict__ v, const int* __restrict__ row_of,
                                 const T* __restrict__ val, long long nnz, int* __restrict__ scol,
                                 int* __restrict__ ocol, T* __restrict__ oval) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= nnz) return;
  scol[p] = (int)k[p];
  ocol[p] = row_of[v[p]];
  oval[p] = val[v[p]];
}

template <typename T>
__global__ void dia_transpose(const int* __restrict__ offset, const T* __restrict__ data, int nd,
                              int stride, int N, int* __restrict__ ooffset, T* __restrict__ odata) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)nd * N) return;
  const int d = (int)(q / N), t = (int)(q - (long long)d * N);
  const int k = offset[d];
  if (t == 0) ooffset[d] = -k;
  const int lo = k < 0 ? -k : 0, hi = (N < N - k) ? N : N - k;
  if (t >= hi - lo) return;
  const int olo = -k < 0 ? k : 0;
  const long long ib = (long long)d * stride - (k < 0 ? (long long)(N - stride) : 0);
  const long long ob = (long long)d * stride - (-k < 0 ? (long long)(N - stride) : 0);
  odata[ob + olo + t] = data[ib + lo + t];
}

template <typename T>
__global__ void ell_col_counts(const T* __restrict__ data, const int* __restrict__ idx,
                               long long slots, int N, int* __restrict__ cnt) {
  const long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (s < slots && nz(data[s])) {
    const int c = idx[s];
    if (c >= 0 && c < N) atomicAdd(cnt + c, 1);
  }
}

// Items in source-row-major order q = j*nc + k; key = column (N for zeros).
template <typename T>
__global__ void ell_t_keys(const T* __restrict__ data, const int* __restrict__ idx, int nc, int N,
                           unsigned long long* __restrict__ keys, unsigned* __restrict__ vals) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)nc * N) return;
  const int j = (int)(q / nc), k = (int)(q - (long long)j * nc);
  const long long s = (long long)k * N + j;
  const int c = idx[s];
  keys[q] = (nz(data[s]) && c >= 0 && c < N) ? (unsigned long long)(unsigned)c
                                                : (unsigned long long)(unsigned)N;
  vals[q] = (unsigned)q;
}

__global__ void keys_to_int(const unsigned long long* __restrict__ k, long long n,
                            int* __restrict__ out) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) out[p] = (int)k[p];
}

template <typename T>
__global__ void ell_t_place(const int* __restrict__ skey, const unsigned* __restrict__ sval,
                            const int* __restrict__ start, const T* __restrict__ data, int nc,
                            int N, int onc, T* __restrict__ odata, int* __restrict__ oidx) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (long long)nc * N) return;
  const int c = skey[p];
  if (c >= N) return;
  const long long rank = p - start[c];
  if (rank >= onc) return;
  const unsigned q = sval[p];
  const int j = (int)(q / nc), k = (int)(q - (unsigned)j * nc);
  odata[rank * N + c] = data[(long long)k * N + j];
  oidx[rank * N + c] = j;
}

static int dt_ok(int dtype, const char* fn) {
  if (dtype == SB_F32 || dtype == SB_F64) return SB_OK;
  set_error("%s: dtype must be SB_F32 or SB_F64", fn);
  return SB_EINVAL;
}

template <typename T>
static int count_nz_impl(const T* v, long long n, long long* count, cudaStream_t st) {
  unsigned long long* d = nullptr;
  int r = scratch_alloc((void**)&d, sizeof(unsigned long long), st);
  if (r) return r;
  SB_CHECK_CUDA(cudaMemsetAsync(d, 0, sizeof(unsigned long long), st));
  count_nz<T><<<std::min<unsigned>(g1(n), (unsigned)sm_count() * 8), kTh, 0, st>>>(v, n, d);
  SB_CHECK_LAUNCH("count_nz");
  unsigned long long h = 0;
  SB_CHECK_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  scratch_free(d, st);
  *count = (long long)h;
  return SB_OK;
}

template <typename T>
static int copy_nz_impl(const int* row_ptr, int N, const int* row, const int* col, const T* val,
                        long long n, int* orow_or_ptr, int* ocol, T* oval, cudaStream_t st) {
  int* pos = nullptr;
  int r = scratch_alloc((void**)&pos, sizeof(int) * (size_t)(n + 1), st);
  if (r) return r;
  nz_flags<T><<<g1(n + 1), kTh, 0, st>>>(val, n, pos);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) r = cuda_status(e, "nz_flags");
  if (!r) r = prim::exclusive_scan(pos, pos, n + 1, st);
  if (!r) {
    scatter_nz_coo<T><<<g1(n), kTh, 0, st>>>(row, col, val, n, pos, row_ptr ? nullptr : orow_or_ptr,
                                              ocol, oval);
    if (row_ptr) rowptr_through<<<g1((long long)N + 1), kTh, 0, st>>>(row_ptr, N, pos, orow_or_ptr);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "copy_nonzeros");
  }
  if (!r && (e = cudaStreamSynchronize(st)) != cudaSuccess) r = cuda_status(e, "copy_nonzeros");
  scratch_free(pos, st);
  return r;
}

template <typename T>
static int dia_nz_impl(const int* offset, const T* data, int nd, int stride, int N, int* count_diags,
                       long long* count, int* ooffset, T* odata, cudaStream_t st) {
  const long long total = (long long)nd * N;
  int* pos = nullptr;
  int r = scratch_alloc((void**)&pos, sizeof(int) * (size_t)(total + 1 + nd + 1), st);
  if (r) return r;
  int* slot = pos + total + 1;
  dia_nz_flags<T><<<g1(total + 1), kTh, 0, st>>>(offset, data, nd, stride, N, pos);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) r = cuda_status(e, "dia_nz_flags");
  if (!r) r = prim::exclusive_scan(pos, pos, total + 1, st);
  if (!r) {
    dia_kept<<<g1(nd + 1), kTh, 0, st>>>(pos, nd, N, slot);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "dia_kept");
  }
  if (!r) r = prim::exclusive_scan(slot, slot, nd + 1, st);
  if (!r && count_diags) {
    int h[2] = {0, 0};
    e = cudaMemcpyAsync(&h[0], slot + nd, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h[1], pos + total, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "count_nonzeros_dia");
    *count_diags = h[0];
    *count = h[1];
  }
  if (!r && odata) {
    int kept = 0;
    e = cudaMemcpyAsync(&kept, slot + nd, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess)
      e = cudaMemsetAsync(odata, 0, sizeof(T) * (size_t)kept * (size_t)stride, st);
    if (e == cudaSuccess) {
      dia_copy_nz<T><<<g1(total), kTh, 0, st>>>(offset, data, nd, stride, N, pos, slot, ooffset,
                                                odata);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "copy_nonzeros_dia");
  }
  scratch_free(pos, st);
  return r;
}

template <typename T>
static int transpose_csr_impl(const int* row_ptr, const int* col, const T* val, int N,
                              long long nnz, int* orow_ptr, int* ocol, T* oval, cudaStream_t st) {
  if (nnz == 0) {
    SB_CHECK_CUDA(cudaMemsetAsync(orow_ptr, 0, sizeof(int) * ((size_t)N + 1), st));
    SB_CHECK_CUDA(cudaStreamSynchronize(st));
    return SB_OK;
  }
  prim::RadixBuffers b;
  void* mem = nullptr;
  const size_t kb = sizeof(unsigned long long) * nnz, vb = sizeof(unsigned) * nnz;
  int r = scratch_alloc(&mem, 2 * kb + 2 * vb + 2 * sizeof(int) * nnz, st);
  if (r) return r;
  char* p = (char*)mem;
  b.k[0] = (unsigned long long*)p;
  b.k[1] = (unsigned long long*)(p + kb);
  b.v[0] = (unsigned*)(p + 2 * kb);
  b.v[1] = (unsigned*)(p + 2 * kb + vb);
  int* row_of = (int*)(p + 2 * kb + 2 * vb);
  int* scol = row_of + nnz;
  prim::expand_rows<<<g1(N), kTh, 0, st>>>(row_ptr, N, row_of);
  col_keys<<<g1(nnz), kTh, 0, st>>>(col, nnz, b.k[0], b.v[0]);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) r = cuda_status(e, "transpose_csr");
  const int ranges[2] = {0, prim::bits_for(N > 0 ? N - 1 : 0)};
  int which = 0;
  if (!r) r = prim::radix_sort_ranges(b, nnz, ranges, 1, &which, st);
  if (!r) {
    transpose_gather<T><<<g1(nnz), kTh, 0, st>>>(b.k[which], b.v[which], row_of, val, nnz, scol,
                                                  ocol, oval);
    prim::row_ptr_from_sorted<<<g1(nnz + 1), kTh, 0, st>>>(scol, nnz, N, orow_ptr);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "transpose_csr");
  }
  scratch_free(mem, st);
  return r;
}

template <typename T>
static int transpose_ell_impl(const T* data, const int* idx, int nc, int N, int onc, T* odata,
                              int* oidx, cudaStream_t st) {
  const long long n = (long long)nc * N;
  SB_CHECK_CUDA(cudaMemsetAsync(odata, 0, sizeof(T) * (size_t)onc * N, st));
  SB_CHECK_CUDA(cudaMemsetAsync(oidx, 0, sizeof(int) * (size_t)onc * N, st));
  if (n == 0) return SB_OK;
  prim::RadixBuffers b;
  void* mem = nullptr;
  const size_t kb = sizeof(unsigned long long) * n, vb = sizeof(unsigned) * n;
  int r = scratch_alloc(&mem, 2 * kb + 2 * vb + sizeof(int) * (n + (size_t)N + 1), st);
  if (r) return r;
  char* p = (char*)mem;
  b.k[0] = (unsigned long long*)p;
  b.k[1] = (unsigned long long*)(p + kb);
  b.v[0] = (unsigned*)(p + 2 * kb);
  b.v[1] = (unsigned*)(p + 2 * kb + vb);
  int* skey = (int*)(p + 2 * kb + 2 * vb);
  int* start = skey + n;
  ell_t_keys<T><<<g1(n), kTh, 0, st>>>(data, idx, nc, N, b.k[0], b.v[0]);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) r = cuda_status(e, "transpose_ell");
  const int ranges[2] = {0, prim::bits_for(N)};
  int which = 0;
  if (!r) r = prim::radix_sort_ranges(b, n, ranges, 1, &which, st);
  if (!r) {
    keys_to_int<<<g1(n), kTh, 0, st>>>(b.k[which], n, skey);
    // start[c] = first sorted position of column c (key N marks zeros)
    prim::row_ptr_from_sorted<<<g1(n + 1), kTh, 0, st>>>(skey, n, N, start);
    ell_t_place<T><<<g1(n), kTh, 0, st>>>(skey, b.v[which], start, data, nc, N, onc, odata, oidx);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "transpose_ell");
  }
  scratch_free(mem, st);
  return r;
}

}  // namespace sb

using namespace sb;

#define SB_DISPATCH(dtype, CALL_F32, CALL_F64) ((dtype) == SB_F32 ? (CALL_F32) : (CALL_F64))

extern "C" {

int sb_count_nonzeros(int dtype, const void* val, int64_t n, int64_t* count, void* stream) {
  SB_TRACE("sb_count_nonzeros");
  int r = dt_ok(dtype, "sb_count_nonzeros");
  if (r) return r;
  SB_REQUIRE(count && n >= 0, "sb_count_nonzeros: bad argument");
  *count = 0;
  if (n == 0) return SB_OK;
  SB_REQUIRE(val, "sb_count_nonzeros: null pointer");
  if ((r = ensure_device())) return r;
  long long c = 0;
  cudaStream_t st = as_stream(stream);
  r = SB_DISPATCH(dtype, count_nz_impl<float>((const float*)val, n, &c, st),
                  count_nz_impl<double>((const double*)val, n, &c, st));
  *count = c;
  return r;
}

int sb_copy_nonzeros_coo(int dtype, const int32_t* row, const int32_t* col, const void* val,
                         int64_t nnz, int32_t* orow, int32_t* ocol, void* oval, void* stream) {
  SB_TRACE("sb_copy_nonzeros_coo");
  int r = dt_ok(dtype, "sb_copy_nonzeros_coo");
  if (r) return r;
  SB_REQUIRE(nnz >= 0 && nnz < 0x7fffffffLL, "sb_copy_nonzeros_coo: bad size");
  if (nnz == 0) return SB_OK;
  SB_REQUIRE(row && col && val && orow && ocol && oval, "sb_copy_nonzeros_coo: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  return SB_DISPATCH(dtype,
                     copy_nz_impl<float>(nullptr, 0, row, col, (const float*)val, nnz, orow, ocol,
                                         (float*)oval, st),
                     copy_nz_impl<double>(nullptr, 0, row, col, (const double*)val, nnz, orow,
                                          ocol, (double*)oval, st));
}

int sb_copy_nonzeros_csr(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                         int32_t N, int64_t nnz, int32_t* orow_ptr, int32_t* ocol, void* oval,
                         void* stream) {
  SB_TRACE("sb_copy_nonzeros_csr");
  int r = dt_ok(dtype, "sb_copy_nonzeros_csr");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nnz >= 0 && nnz < 0x7fffffffLL, "sb_copy_nonzeros_csr: bad size");
  SB_REQUIRE(row_ptr && orow_ptr && (nnz == 0 || (col && val && ocol && oval)),
             "sb_copy_nonzeros_csr: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  return SB_DISPATCH(dtype,
                     copy_nz_impl<float>(row_ptr, N, nullptr, col, (const float*)val, nnz,
                                         orow_ptr, ocol, (float*)oval, st),
                     copy_nz_impl<double>(row_ptr, N, nullptr, col, (const double*)val, nnz,
                                          orow_ptr, ocol, (double*)oval, st));
}

int sb_count_nonzeros_dia(int dtype, const int32_t* offset, const void* data, int32_t nd,
                          int32_t stride, int32_t N, int32_t* count_diags, int64_t* count,
                          void* stream) {
  SB_TRACE("sb_count_nonzeros_dia");
  int r = dt_ok(dtype, "sb_count_nonzeros_dia");
  if (r) return r;
  SB_REQUIRE(count_diags && count && nd >= 0 && N >= 0 && stride >= N,
             "sb_count_nonzeros_dia: bad argument");
  *count_diags = 0;
  *count = 0;
  if (nd == 0 || N == 0) return SB_OK;
  SB_REQUIRE(offset && data, "sb_count_nonzeros_dia: null pointer");
  if ((r = ensure_device())) return r;
  long long c = 0;
  cudaStream_t st = as_stream(stream);
  r = SB_DISPATCH(dtype,
                  dia_nz_impl<float>(offset, (const float*)data, nd, stride, N, count_diags, &c,
                                     nullptr, nullptr, st),
                  dia_nz_impl<double>(offset, (const double*)data, nd, stride, N, count_diags, &c,
                                      nullptr, nullptr, st));
  *count = c;
  return r;
}

int sb_copy_nonzeros_dia(int dtype, const int32_t* offset, const void* data, int32_t nd,
                         int32_t stride, int32_t N, int32_t* ooffset, void* odata, void* stream) {
  SB_TRACE("sb_copy_nonzeros_dia");
  int r = dt_ok(dtype, "sb_copy_nonzeros_dia");
  if (r) return r;
  SB_REQUIRE(nd >= 0 && N >= 0 && stride >= N, "sb_copy_nonzeros_dia: bad size");
  if (nd == 0 || N == 0) return SB_OK;
  SB_REQUIRE(offset && data && ooffset && odata, "sb_copy_nonzeros_dia: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  return SB_DISPATCH(dtype,
                     dia_nz_impl<float>(offset, (const float*)data, nd, stride, N, nullptr,
                                        nullptr, ooffset, (float*)odata, st),
                     dia_nz_impl<double>(offset, (const double*)data, nd, stride, N, nullptr,
                                         nullptr, ooffset, (double*)odata, st));
}

int sb_count_nonzeros_ell(int dtype, const void* data, int32_t nc, int32_t N, int32_t* count_cols,
                          int64_t* count, void* stream) {
  SB_TRACE("sb_count_nonzeros_ell");
  int r = dt_ok(dtype, "sb_count_nonzeros_ell");
  if (r) return r;
  SB_REQUIRE(count_cols && count && nc >= 0 && N >= 0, "sb_count_nonzeros_ell: bad argument");
  *count_cols = 0;
  *count = 0;
  if (nc == 0 || N == 0) return SB_OK;
  SB_REQUIRE(data, "sb_count_nonzeros_ell: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  // layout: [u64 sum][int max][int pad][int counts[N]] (8-byte aligned sum)
  unsigned long long* sum = nullptr;
  if ((r = scratch_alloc((void**)&sum, sizeof(unsigned long long) + sizeof(int) * ((size_t)N + 2),
                         st)))
    return r;
  int* mx = (int*)(sum + 1);
  int* cnt = mx + 2;
  SB_CHECK_CUDA(cudaMemsetAsync(sum, 0, sizeof(unsigned long long) + 2 * sizeof(int), st));
  if (dtype == SB_F32) ell_row_counts<float><<<g1(N), kTh, 0, st>>>((const float*)data, nc, N, cnt);
  else ell_row_counts<double><<<g1(N), kTh, 0, st>>>((const double*)data, nc, N, cnt);
  max_sum<<<std::min<unsigned>(g1(N), (unsigned)sm_count() * 8), kTh, 0, st>>>(cnt, N, mx, sum);
  SB_CHECK_LAUNCH("count_nonzeros_ell");
  unsigned long long s = 0;
  int h[1] = {0};
  SB_CHECK_CUDA(cudaMemcpyAsync(&s, sum, sizeof(s), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaMemcpyAsync(h, mx, sizeof(int), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  scratch_free(sum, st);
  *count_cols = h[0];
  *count = (int64_t)s;
  return SB_OK;
}

int sb_copy_nonzeros_ell(int dtype, const void* data, const int32_t* indices, int32_t nc,
                         int32_t N, int32_t out_nc, void* odata, int32_t* oindices, void* stream) {
  SB_TRACE("sb_copy_nonzeros_ell");
  int r = dt_ok(dtype, "sb_copy_nonzeros_ell");
  if (r) return r;
  SB_REQUIRE(nc >= 0 && N >= 0 && out_nc >= 0, "sb_copy_nonzeros_ell: bad size");
  if (N == 0 || out_nc == 0) return SB_OK;
  SB_REQUIRE(data && indices && odata && oindices, "sb_copy_nonzeros_ell: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  if (dtype == SB_F32)
    ell_copy_nz<float><<<g1(N), kTh, 0, st>>>((const float*)data, indices, nc, N, out_nc,
                                             (float*)odata, oindices);
  else
    ell_copy_nz<double><<<g1(N), kTh, 0, st>>>((const double*)data, indices, nc, N, out_nc,
                                              (double*)odata, oindices);
  SB_CHECK_LAUNCH("copy_nonzeros_ell");
  return SB_OK;
}

int sb_transpose_coo(int dtype, const int32_t* row, const int32_t* col, const void* val,
                     int64_t nnz, int32_t* orow, int32_t* ocol, void* oval, void* stream) {
  SB_TRACE("sb_transpose_coo");
  int r = dt_ok(dtype, "sb_transpose_coo");
  if (r) return r;
  SB_REQUIRE(nnz >= 0, "sb_transpose_coo: bad size");
  if (nnz == 0) return SB_OK;
  SB_REQUIRE(row && col && val && orow && ocol && oval, "sb_transpose_coo: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  SB_CHECK_CUDA(cudaMemcpyAsync(ocol, row, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, st));
  SB_CHECK_CUDA(cudaMemcpyAsync(orow, col, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, st));
  SB_CHECK_CUDA(cudaMemcpyAsync(oval, val, dtype_size(dtype) * nnz, cudaMemcpyDeviceToDevice, st));
  return SB_OK;
}

int sb_transpose_csr(int dtype, const int32_t* row_ptr, const int32_t* col, const void* val,
                     int32_t N, int64_t nnz, int32_t* orow_ptr, int32_t* ocol, void* oval,
                     void* stream) {
  SB_TRACE("sb_transpose_csr");
  int r = dt_ok(dtype, "sb_transpose_csr");
  if (r) return r;
  SB_REQUIRE(N >= 0 && nnz >= 0 && nnz < 0x7fffffffLL, "sb_transpose_csr: bad size");
  SB_REQUIRE(row_ptr && orow_ptr && (nnz == 0 || (col && val && ocol && oval)),
             "sb_transpose_csr: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  return SB_DISPATCH(dtype,
                     transpose_csr_impl<float>(row_ptr, col, (const float*)val, N, nnz, orow_ptr,
                                               ocol, (float*)oval, st),
                     transpose_csr_impl<double>(row_ptr, col, (const double*)val, N, nnz,
                                                orow_ptr, ocol, (double*)oval, st));
}

int sb_transpose_dia(int dtype, const int32_t* offset, const void* data, int32_t nd,
                     int32_t stride, int32_t N, int32_t* ooffset, void* odata, void* stream) {
  SB_TRACE("sb_transpose_dia");
  int r = dt_ok(dtype, "sb_transpose_dia");
  if (r) return r;
  SB_REQUIRE(nd >= 0 && N >= 0 && stride >= N, "sb_transpose_dia: bad size");
  if (nd == 0 || N == 0) return SB_OK;
  SB_REQUIRE(offset && data && ooffset && odata, "sb_transpose_dia: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  SB_CHECK_CUDA(cudaMemsetAsync(odata, 0, dtype_size(dtype) * (size_t)nd * stride, st));
  const long long total = (long long)nd * N;
  if (dtype == SB_F32)
    dia_transpose<float><<<g1(total), kTh, 0, st>>>(offset, (const float*)data, nd, stride, N,
                                                    ooffset, (float*)odata);
  else
    dia_transpose<double><<<g1(total), kTh, 0, st>>>(offset, (const double*)data, nd, stride, N,
                                                     ooffset, (double*)odata);
  SB_CHECK_LAUNCH("transpose_dia");
  return SB_OK;
}

int sb_count_transpose_cols_ell(int dtype, const void* data, const int32_t* indices, int32_t nc,
                                int32_t N, int32_t* count_cols, void* stream) {
  SB_TRACE("sb_count_transpose_cols_ell");
  int r = dt_ok(dtype, "sb_count_transpose_cols_ell");
  if (r) return r;
  SB_REQUIRE(count_cols && nc >= 0 && N >= 0, "sb_count_transpose_cols_ell: bad argument");
  *count_cols = 0;
  if (nc == 0 || N == 0) return SB_OK;
  SB_REQUIRE(data && indices, "sb_count_transpose_cols_ell: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  int* cnt = nullptr;
  if ((r = scratch_alloc((void**)&cnt, sizeof(int) * ((size_t)N + 2), st))) return r;
  SB_CHECK_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * ((size_t)N + 2), st));
  const long long slots = (long long)nc * N;
  if (dtype == SB_F32)
    ell_col_counts<float><<<g1(slots), kTh, 0, st>>>((const float*)data, indices, slots, N, cnt);
  else
    ell_col_counts<double><<<g1(slots), kTh, 0, st>>>((const double*)data, indices, slots, N, cnt);
  max_sum<<<std::min<unsigned>(g1(N), (unsigned)sm_count() * 8), kTh, 0, st>>>(cnt, N, cnt + N,
                                                                              nullptr);
  SB_CHECK_LAUNCH("count_transpose_cols_ell");
  SB_CHECK_CUDA(cudaMemcpyAsync(count_cols, cnt + N, sizeof(int), cudaMemcpyDeviceToHost, st));
  SB_CHECK_CUDA(cudaStreamSynchronize(st));
  scratch_free(cnt, st);
  return SB_OK;
}

int sb_transpose_ell(int dtype, const void* data, const int32_t* indices, int32_t nc, int32_t N,
                     int32_t out_nc, void* odata, int32_t* oindices, void* stream) {
  SB_TRACE("sb_transpose_ell");
  int r = dt_ok(dtype, "sb_transpose_ell");
  if (r) return r;
  SB_REQUIRE(nc >= 0 && N >= 0 && out_nc >= 0, "sb_transpose_ell: bad size");
  SB_REQUIRE((long long)nc * N < 0x7fffffffLL, "sb_transpose_ell: too many slots");
  if (N == 0 || out_nc == 0) return SB_OK;
  SB_REQUIRE(data && indices && odata && oindices, "sb_transpose_ell: null pointer");
  if ((r = ensure_device())) return r;
  cudaStream_t st = as_stream(stream);
  return SB_DISPATCH(dtype,
                     transpose_ell_impl<float>((const float*)data, indices, nc, N, out_nc,
                                               (float*)odata, oindices, st),
                     transpose_ell_impl<double>((const double*)data, indices, nc, N, out_nc,
                                                (double*)odata, oindices, st));
}

}  // extern "C"
