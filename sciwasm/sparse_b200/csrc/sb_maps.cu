// sb_maps.cu -- element-wise maps on the value arrays, as the reference's
// *_coo (COO and CSR values), *_dia (in-band slots only) and *_ell (every
// slot, padding included) wasm kernels (src/sequential/src/sparse_opt_32.wat:
// 597-1699, 2137-4976, 4977-6346).  in == out gives the in-place (self_*)
// forms.  f32 transcendentals are evaluated in double and rounded to f32,
// which is what the reference's imported JavaScript Math functions do
// (:5-9); deg2rad / rad2deg use fl(p / 180) with p rounded to the value type
// (the reference passes Math.PI as the value-typed parameter).  Sign: the COO
// kernels map v > 0 to 1 and everything else to -1; the DIA/ELL kernels map
// 0 to 0 (and NaN to -1).
#include <algorithm>

#include "sb_common.cuh"

namespace sb {

constexpr int kMT = 256;

template <typename T> struct mops;
template <> struct mops<float> {
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ float sqrt_(float a) { return __fsqrt_rn(a); }
};
template <> struct mops<double> {
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ double sqrt_(double a) { return __dsqrt_rn(a); }
};

template <typename T, int KIND>
__device__ __forceinline__ T map_one(int op, T p, T k180, T v) {
  switch (op) {
    case SB_MAP_EXPM1: return (T)expm1((double)v);
    case SB_MAP_LOG1P: return (T)log1p((double)v);
    case SB_MAP_SIN: return (T)sin((double)v);
    case SB_MAP_TAN: return (T)tan((double)v);
    case SB_MAP_POW: return (T)pow((double)v, (double)p);
    case SB_MAP_DEG2RAD: return mops<T>::mul(v, k180);
    case SB_MAP_RAD2DEG: return mops<T>::div(v, k180);
    case SB_MAP_SIGN:
      if (KIND == 1 && v == (T)0) return (T)0;
      return v > (T)0 ? (T)1 : (T)-1;
    case SB_MAP_ABS: return fabs(v);
    case SB_MAP_NEG: return -v;
    case SB_MAP_SQRT: return mops<T>::sqrt_(v);
    case SB_MAP_CEIL: return ceil(v);
    case SB_MAP_FLOOR: return floor(v);
    case SB_MAP_TRUNC: return trunc(v);
    case SB_MAP_NEAREST: return rint(v);
    case SB_MAP_MULTIPLY: return mops<T>::mul(v, p);
  }
  return v;
}

template <typename T, int KIND>
__global__ void map_kernel(int op, T p, T k180, const T* __restrict__ in, T* __restrict__ out,
                           long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = map_one<T, KIND>(op, p, k180, in[i]);
}

// DIA: in-band slots are mapped; out-of-band slots of a separate output are
// zeroed (the reference leaves them as the allocator returned them).
template <typename T>
__global__ void map_dia_kernel(int op, T p, T k180, const int* __restrict__ offset,
                               const T* in, T* out, int nd, int stride, int N, int zero_rest) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (long long)nd * stride) return;
  const int d = (int)(q / stride), s = (int)(q - (long long)d * stride);
  const int k = offset[d];
  const int row = s + (k < 0 ? N - stride : 0);
  const bool inband = row >= 0 && row < N && (unsigned)(row + k) < (unsigned)N;
  if (inband) out[q] = map_one<T, 1>(op, p, k180, in[q]);
  else if (zero_rest) out[q] = (T)0;
}

static int map_check(int dtype, int op, const char* fn) {
  if (dtype != SB_F32 && dtype != SB_F64) {
    set_error("%s: dtype must be SB_F32 or SB_F64", fn);
    return SB_EINVAL;
  }
  if (op < 0 || op > SB_MAP_MULTIPLY) {
    set_error("%s: unknown map op %d", fn, op);
    return SB_EINVAL;
  }
  return ensure_device();
}

template <typename T, int KIND>
static int launch_map(int op, double p, const void* in, void* out, long long n, cudaStream_t st) {
  const T pt = (T)p;
  T k180;
  if (sizeof(T) == 4) k180 = (T)((float)pt / 180.0f);
  else k180 = (T)(p / 180.0);
  const long long g = std::min<long long>((n + kMT - 1) / kMT, (long long)sm_count() * 16);
  map_kernel<T, KIND><<<(unsigned)std::max(1LL, g), kMT, 0, st>>>(op, pt, k180, (const T*)in,
                                                                  (T*)out, n);
  SB_CHECK_LAUNCH("map_kernel");
  return SB_OK;
}

template <typename A, typename B> __device__ __forceinline__ B conv(A v) { return (B)v; }
template <> __device__ __forceinline__ __nv_bfloat16 conv(float v) { return __float2bfloat16_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 conv(double v) {
  return __float2bfloat16_rn(__double2float_rn(v));
}
template <> __device__ __forceinline__ float conv(__nv_bfloat16 v) { return __bfloat162float(v); }
template <> __device__ __forceinline__ double conv(__nv_bfloat16 v) {
  return (double)__bfloat162float(v);
}
template <> __device__ __forceinline__ float conv(double v) { return __double2float_rn(v); }

template <typename A, typename B>
__global__ void convert_kernel(const A* __restrict__ in, B* __restrict__ out, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    out[i] = conv<A, B>(in[i]);
}

template <typename A>
static int convert_from(const A* in, int dst, void* out, long long n, cudaStream_t st) {
  const unsigned g = (unsigned)std::min<long long>((n + kMT - 1) / kMT, (long long)sm_count() * 16);
  if (dst == SB_F32) convert_kernel<A, float><<<g, kMT, 0, st>>>(in, (float*)out, n);
  else if (dst == SB_F64) convert_kernel<A, double><<<g, kMT, 0, st>>>(in, (double*)out, n);
  else convert_kernel<A, __nv_bfloat16><<<g, kMT, 0, st>>>(in, (__nv_bfloat16*)out, n);
  SB_CHECK_LAUNCH("convert_kernel");
  return SB_OK;
}

}  // namespace sb

using namespace sb;

extern "C" {

int sb_convert_values(int src_dtype, const void* src, int dst_dtype, void* dst, int64_t n,
                      void* stream) {
  SB_TRACE("sb_convert_values");
  const bool ok = (src_dtype >= SB_F32 && src_dtype <= SB_BF16) &&
                  (dst_dtype >= SB_F32 && dst_dtype <= SB_BF16);
  SB_REQUIRE(ok, "sb_convert_values: dtypes must be SB_F32, SB_F64 or SB_BF16");
  SB_REQUIRE(n >= 0, "sb_convert_values: negative size");
  if (n == 0) return SB_OK;
  SB_REQUIRE(src && dst, "sb_convert_values: null pointer");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  if (src_dtype == SB_F32) return convert_from<float>((const float*)src, dst_dtype, dst, n, st);
  if (src_dtype == SB_F64) return convert_from<double>((const double*)src, dst_dtype, dst, n, st);
  return convert_from<__nv_bfloat16>((const __nv_bfloat16*)src, dst_dtype, dst, n, st);
}

int sb_map_coo(int dtype, int op, double p, const void* in, void* out, int64_t n, void* stream) {
  SB_TRACE("sb_map_coo");
  int r = map_check(dtype, op, "sb_map_coo");
  if (r) return r;
  SB_REQUIRE(n >= 0, "sb_map_coo: negative size");
  if (n == 0) return SB_OK;
  SB_REQUIRE(in && out, "sb_map_coo: null pointer");
  cudaStream_t st = as_stream(stream);
  return dtype == SB_F32 ? launch_map<float, 0>(op, p, in, out, n, st)
                         : launch_map<double, 0>(op, p, in, out, n, st);
}

int sb_map_ell(int dtype, int op, double p, const void* in, void* out, int32_t ncols, int32_t N,
               void* stream) {
  SB_TRACE("sb_map_ell");
  int r = map_check(dtype, op, "sb_map_ell");
  if (r) return r;
  SB_REQUIRE(ncols >= 0 && N >= 0, "sb_map_ell: negative size");
  const long long n = (long long)ncols * N;
  if (n == 0) return SB_OK;
  SB_REQUIRE(in && out, "sb_map_ell: null pointer");
  cudaStream_t st = as_stream(stream);
  return dtype == SB_F32 ? launch_map<float, 1>(op, p, in, out, n, st)
                         : launch_map<double, 1>(op, p, in, out, n, st);
}

int sb_map_dia(int dtype, int op, double p, const int32_t* offset, const void* in, void* out,
               int32_t ndiags, int32_t stride, int32_t N, void* stream) {
  SB_TRACE("sb_map_dia");
  int r = map_check(dtype, op, "sb_map_dia");
  if (r) return r;
  SB_REQUIRE(ndiags >= 0 && N >= 0 && stride >= N, "sb_map_dia: bad size");
  const long long n = (long long)ndiags * stride;
  if (n == 0) return SB_OK;
  SB_REQUIRE(offset && in && out, "sb_map_dia: null pointer");
  cudaStream_t st = as_stream(stream);
  const unsigned g = (unsigned)((n + kMT - 1) / kMT);
  const int zero_rest = in != out;
  if (dtype == SB_F32) {
    const float pt = (float)p;
    map_dia_kernel<float><<<g, kMT, 0, st>>>(op, pt, pt / 180.0f, offset, (const float*)in,
                                             (float*)out, ndiags, stride, N, zero_rest);
  } else {
    map_dia_kernel<double><<<g, kMT, 0, st>>>(op, p, p / 180.0, offset, (const double*)in,
                                              (double*)out, ndiags, stride, N, zero_rest);
  }
  SB_CHECK_LAUNCH("map_dia_kernel");
  return SB_OK;
}

}  // extern "C"
