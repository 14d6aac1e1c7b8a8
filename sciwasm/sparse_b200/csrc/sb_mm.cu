// sb_mm.cu -- Matrix Market input: the reference's mmread / create_COO_from_MM
// / create_LCOO_from_MM (src/sequential/src/sparse32.js:1889-2172).
//
// The text is parsed on the host (the header, then the entry lines split
// across threads at line boundaries); the entries go to the device as
// 1-based (row, col, value) arrays, where one kernel counts what each entry
// produces under the reference's rules (explicit zeros dropped, off-diagonal
// entries of "symmetric" files mirrored, or only the strictly lower part plus
// a unit diagonal for the triangular-solve input), a scan gives every entry
// its output slot, a second kernel writes the entries there, and a stable
// radix sort by (row, col) replaces the reference's quick_sort_COO.
#include <algorithm>
#include <atomic>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <thread>
#include <vector>

#include "sb_common.cuh"
#include "sb_prims.cuh"

namespace sb {
namespace {

constexpr int kT = 256;
constexpr long long kMaxEntries = 1LL << 27;  // the reference's allocation limits
constexpr long long kMaxNnz = 1LL << 28;

unsigned grid_n(long long n) {
  const long long g = (n + kT - 1) / kT;
  return (unsigned)std::max(1LL, std::min(g, 0x7fffffffLL));
}

// ---------------------------------------------------------------- host parse

bool same_word(const char* a, size_t n, const char* b) {
  if (strlen(b) != n) return false;
  for (size_t i = 0; i < n; ++i)
    if (tolower((unsigned char)a[i]) != b[i]) return false;
  return true;
}

// Whitespace-separated tokens of [p, e).
int split_tokens(const char* p, const char* e, const char** tok, size_t* len, int cap) {
  int n = 0;
  while (p < e && n < cap) {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
    if (p >= e) break;
    const char* s = p;
    while (p < e && *p != ' ' && *p != '\t' && *p != '\r') ++p;
    tok[n] = s;
    len[n] = (size_t)(p - s);
    ++n;
  }
  return n;
}

bool blank(const char* p, const char* e) {
  for (; p < e; ++p)
    if (*p != ' ' && *p != '\t' && *p != '\r') return false;
  return true;
}

// An entry line is neither blank nor a '%' comment.
bool entry_line(const char* p, const char* e) { return p < e && *p != '%' && !blank(p, e); }

// Parses "row col [value ...]" of one entry line; false when malformed.
bool parse_entry(const char* p, const char* e, bool pattern, long long nrows, long long ncols,
                 int32_t* r, int32_t* c, double* v) {
  char buf[256];
  const size_t n = std::min((size_t)(e - p), sizeof(buf) - 1);
  memcpy(buf, p, n);
  buf[n] = 0;
  char* q = buf;
  char* end = nullptr;
  const long long rr = strtoll(q, &end, 10);
  if (end == q) return false;
  q = end;
  const long long cc = strtoll(q, &end, 10);
  if (end == q) return false;
  q = end;
  if (rr < 1 || rr > nrows || cc < 1 || cc > ncols) return false;
  *r = (int32_t)rr;
  *c = (int32_t)cc;
  if (!pattern) {
    const double x = strtod(q, &end);
    if (end == q) return false;
    *v = x;
  }
  return true;
}

// ---------------------------------------------------------------- device

// What entry n produces: 0, 1 or 2 COO entries.
__device__ __forceinline__ int mm_count(int32_t r, int32_t c, double v, bool pattern,
                                        bool symmetric, bool lower) {
  if (!pattern && !(v < 0 || v > 0)) return 0;  // explicit zero (or NaN): dropped
  if (!lower) return (symmetric && r != c) ? 2 : 1;
  if (r > c) return 1;
  return (symmetric && r < c) ? 1 : 0;
}

__global__ void mm_count_kernel(const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                                const double* __restrict__ val, long long n, bool pattern,
                                bool symmetric, bool lower, int* __restrict__ count) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    count[i] = mm_count(row[i], col[i], pattern ? 1.0 : val[i], pattern, symmetric, lower);
}

template <typename T>
__global__ void mm_write_kernel(const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                                const double* __restrict__ val, long long n, bool pattern,
                                bool symmetric, bool lower, const int* __restrict__ offset,
                                long long ndiag_at, long long nrows, int32_t* __restrict__ orow,
                                int32_t* __restrict__ ocol, T* __restrict__ oval) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int32_t r = row[i], c = col[i];
    const double v = pattern ? 1.0 : val[i];
    const int k = mm_count(r, c, v, pattern, symmetric, lower);
    if (!k) continue;
    const long long o = offset[i];
    if (!lower) {
      orow[o] = r - 1;
      ocol[o] = c - 1;
      oval[o] = (T)v;
      if (k == 2) {
        orow[o + 1] = c - 1;
        ocol[o + 1] = r - 1;
        oval[o + 1] = (T)v;
      }
    } else {
      orow[o] = (r > c ? r : c) - 1;
      ocol[o] = (r > c ? c : r) - 1;
      oval[o] = (T)v;
    }
  }
  if (lower)  // the unit diagonal after the off-diagonal entries
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nrows;
         i += (long long)gridDim.x * blockDim.x) {
      orow[ndiag_at + i] = (int32_t)i;
      ocol[ndiag_at + i] = (int32_t)i;
      oval[ndiag_at + i] = (T)1.0;
    }
}

__global__ void mm_pack_keys(const int32_t* __restrict__ row, const int32_t* __restrict__ col,
                             long long n, unsigned long long* __restrict__ key,
                             unsigned* __restrict__ pos) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    key[i] = ((unsigned long long)(unsigned)row[i] << 32) | (unsigned)col[i];
    pos[i] = (unsigned)i;
  }
}

template <typename T>
__global__ void mm_unpack(const unsigned long long* __restrict__ key,
                          const unsigned* __restrict__ pos, const T* __restrict__ vin, long long n,
                          int32_t* __restrict__ orow, int32_t* __restrict__ ocol,
                          T* __restrict__ oval) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    orow[i] = (int32_t)(key[i] >> 32);
    ocol[i] = (int32_t)(key[i] & 0xffffffffu);
    oval[i] = vin[pos[i]];
  }
}

template <typename T>
int mm_coo_impl(bool lower, const sb_mm_header* h, const int32_t* row, const int32_t* col,
                const double* val, int32_t* orow, int32_t* ocol, T* oval, int64_t* nnz,
                cudaStream_t st) {
  const long long n = h->nentries;
  const bool pattern = h->field == SB_MM_PATTERN, symmetric = h->symmetric != 0;
  const long long nrows = lower ? h->nrows : 0;
  int* cnt = nullptr;
  int r = scratch_alloc((void**)&cnt, sizeof(int) * (size_t)(2 * n + 2), st);
  if (r) return r;
  int* off = cnt + n + 1;
  long long total = 0;
  if (n > 0) {
    mm_count_kernel<<<std::min(grid_n(n), 4096u), kT, 0, st>>>(row, col, val, n, pattern,
                                                               symmetric, lower, cnt);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "mm_count_kernel");
    if (!r) r = prim::exclusive_scan(cnt, off, n, st);
    int last[2] = {0, 0};
    if (!r) {
      e = cudaMemcpyAsync(&last[0], cnt + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(&last[1], off + n - 1, sizeof(int), cudaMemcpyDeviceToHost, st);
      if (e == cudaSuccess) e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) r = cuda_status(e, "sb_mm_coo");
    }
    total = (long long)last[0] + last[1];
  }
  const long long offdiag = total;
  total += nrows;
  if (!r && total > kMaxNnz) {
    set_error("sb_mm_coo: %lld nonzeros exceed the limit of 2^28", total);
    r = SB_EINVAL;
  }
  *nnz = total;
  if (r || !orow || total == 0) {
    scratch_free(cnt, st);
    return r;
  }
  // entries (unsorted) into a scratch copy, then the stable sort into the output
  const size_t kb = sizeof(unsigned long long) * (size_t)total;
  const size_t pb = sizeof(unsigned) * (size_t)total;
  const size_t vb = sizeof(T) * (size_t)total;
  void* mem = nullptr;
  if ((r = scratch_alloc(&mem, 2 * kb + 2 * pb + vb + 2 * sizeof(int32_t) * (size_t)total, st))) {
    scratch_free(cnt, st);
    return r;
  }
  char* p = (char*)mem;
  prim::RadixBuffers b;
  b.k[0] = (unsigned long long*)p;
  b.k[1] = (unsigned long long*)(p + kb);
  b.v[0] = (unsigned*)(p + 2 * kb);
  b.v[1] = (unsigned*)(p + 2 * kb + pb);
  T* tval = (T*)(p + 2 * kb + 2 * pb);
  int32_t* trow = (int32_t*)(p + 2 * kb + 2 * pb + vb);
  int32_t* tcol = trow + total;
  const unsigned g = std::min(grid_n(std::max(n, nrows)), 4096u);
  mm_write_kernel<T><<<g, kT, 0, st>>>(row, col, val, n, pattern, symmetric, lower, off, offdiag,
                                       nrows, trow, tcol, tval);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) r = cuda_status(e, "mm_write_kernel");
  if (!r) {
    mm_pack_keys<<<std::min(grid_n(total), 4096u), kT, 0, st>>>(trow, tcol, total, b.k[0],
                                                                b.v[0]);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "mm_pack_keys");
  }
  int which = 0;
  if (!r) {
    const int rb = prim::bits_for(h->nrows > 0 ? h->nrows - 1 : 0);
    const int cb = prim::bits_for(h->ncols > 0 ? h->ncols - 1 : 0);
    const int ranges[4] = {0, cb, 32, 32 + rb};
    r = prim::radix_sort_ranges(b, total, ranges, 2, &which, st);
  }
  if (!r) {
    mm_unpack<T><<<std::min(grid_n(total), 4096u), kT, 0, st>>>(b.k[which], b.v[which], tval,
                                                               total, orow, ocol, oval);
    e = cudaGetLastError();
    if (e != cudaSuccess) r = cuda_status(e, "mm_unpack");
  }
  if (!r) {
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) r = cuda_status(e, "sb_mm_coo");
  }
  scratch_free(mem, st);
  scratch_free(cnt, st);
  return r;
}

}  // namespace
}  // namespace sb

using namespace sb;

extern "C" {

int sb_mm_read_header(const char* text, size_t len, sb_mm_header* h) {
  SB_TRACE("sb_mm_read_header");
  SB_REQUIRE(text && h, "sb_mm_read_header: null argument");
  memset(h, 0, sizeof(*h));
  const char* p = text;
  const char* end = text + len;
  // banner: %%MatrixMarket matrix coordinate <field> <symmetry>
  const char* le = (const char*)memchr(p, '\n', (size_t)(end - p));
  if (!le) le = end;
  const char* tok[8];
  size_t tl[8];
  const int nt = split_tokens(p, le, tok, tl, 8);
  SB_REQUIRE(nt >= 5 && same_word(tok[0], tl[0], "%%matrixmarket"),
             "sb_mm_read_header: not a Matrix Market banner");
  SB_REQUIRE(same_word(tok[2], tl[2], "coordinate"),
             "sb_mm_read_header: only the coordinate format is supported");
  h->field = same_word(tok[3], tl[3], "real")      ? SB_MM_REAL
             : same_word(tok[3], tl[3], "integer") ? SB_MM_INTEGER
             : same_word(tok[3], tl[3], "pattern") ? SB_MM_PATTERN
             : same_word(tok[3], tl[3], "complex") ? SB_MM_COMPLEX
                                                   : -1;
  SB_REQUIRE(h->field >= 0, "sb_mm_read_header: unknown field");
  h->symmetric = same_word(tok[4], tl[4], "symmetric") ? 1 : 0;
  // comments and blank lines, then "nrows ncols nentries"
  p = le < end ? le + 1 : end;
  while (p < end) {
    le = (const char*)memchr(p, '\n', (size_t)(end - p));
    if (!le) le = end;
    if (entry_line(p, le)) break;
    p = le < end ? le + 1 : end;
  }
  SB_REQUIRE(p < end, "sb_mm_read_header: missing size line");
  const int ns = split_tokens(p, le, tok, tl, 8);
  SB_REQUIRE(ns >= 3, "sb_mm_read_header: malformed size line");
  long long v[3];
  for (int i = 0; i < 3; ++i) {
    char buf[32];
    const size_t n = std::min(tl[i], sizeof(buf) - 1);
    memcpy(buf, tok[i], n);
    buf[n] = 0;
    char* q = nullptr;
    v[i] = strtoll(buf, &q, 10);
    SB_REQUIRE(q != buf && v[i] >= 0, "sb_mm_read_header: malformed size line");
  }
  SB_REQUIRE(v[0] <= 0x7fffffffLL && v[1] <= 0x7fffffffLL,
             "sb_mm_read_header: dimensions exceed int32");
  if (v[2] > kMaxEntries) {
    set_error("sb_mm_read_header: %lld entries exceed the limit of 2^27", v[2]);
    return SB_EINVAL;
  }
  h->nrows = v[0];
  h->ncols = v[1];
  h->nentries = v[2];
  h->data_offset = (int64_t)((le < end ? le + 1 : end) - text);
  return SB_OK;
}

int sb_mm_read_entries(const char* text, size_t len, const sb_mm_header* h, int32_t* row,
                       int32_t* col, double* val, int32_t nthreads) {
  SB_TRACE("sb_mm_read_entries");
  SB_REQUIRE(text && h, "sb_mm_read_entries: null argument");
  SB_REQUIRE(h->nentries == 0 || (row && col), "sb_mm_read_entries: null output");
  const bool pattern = h->field == SB_MM_PATTERN;
  SB_REQUIRE(pattern || h->nentries == 0 || val, "sb_mm_read_entries: null value output");
  SB_REQUIRE(h->data_offset >= 0 && (size_t)h->data_offset <= len,
             "sb_mm_read_entries: bad data offset");
  const char* base = text + h->data_offset;
  const char* end = text + len;
  int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
  const size_t bytes = (size_t)(end - base);
  nt = (int)std::max<size_t>(1, std::min<size_t>((size_t)nt, bytes / (1 << 16) + 1));
  // chunk boundaries at line starts
  std::vector<const char*> cut(nt + 1);
  cut[0] = base;
  cut[nt] = end;
  for (int t = 1; t < nt; ++t) {
    const char* q = base + bytes * t / nt;
    if (q < cut[t - 1]) q = cut[t - 1];
    const char* nl = (const char*)memchr(q, '\n', (size_t)(end - q));
    cut[t] = nl ? nl + 1 : end;
  }
  std::vector<long long> lines(nt + 1, 0);
  auto count = [&](int t) {
    long long c = 0;
    for (const char* p = cut[t]; p < cut[t + 1];) {
      const char* le = (const char*)memchr(p, '\n', (size_t)(cut[t + 1] - p));
      if (!le) le = cut[t + 1];
      if (entry_line(p, le)) ++c;
      p = le + 1;
    }
    lines[t + 1] = c;
  };
  std::atomic<long long> bad{-1};
  auto parse = [&](int t) {
    long long j = lines[t];
    for (const char* p = cut[t]; p < cut[t + 1];) {
      const char* le = (const char*)memchr(p, '\n', (size_t)(cut[t + 1] - p));
      if (!le) le = cut[t + 1];
      if (entry_line(p, le)) {
        double v = 0.0;
        if (!parse_entry(p, le, pattern, h->nrows, h->ncols, &row[j], &col[j], &v)) {
          long long expect = -1;
          bad.compare_exchange_strong(expect, j);
        } else if (!pattern) {
          val[j] = v;
        }
        ++j;
      }
      p = le + 1;
    }
  };
  {
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(count, t);
    count(0);
    for (auto& x : th) x.join();
  }
  for (int t = 0; t < nt; ++t) lines[t + 1] += lines[t];
  if (lines[nt] != h->nentries) {
    set_error("sb_mm_read_entries: %lld entry lines, the size line says %lld", lines[nt],
              (long long)h->nentries);
    return SB_EINVAL;
  }
  {
    std::vector<std::thread> th;
    for (int t = 1; t < nt; ++t) th.emplace_back(parse, t);
    parse(0);
    for (auto& x : th) x.join();
  }
  if (bad.load() >= 0) {
    set_error("sb_mm_read_entries: entry %lld is malformed or out of range", bad.load() + 1);
    return SB_EINVAL;
  }
  return SB_OK;
}

int sb_mm_coo(int dtype, int lower, const sb_mm_header* h, const int32_t* row,
              const int32_t* col, const double* val, int32_t* out_row, int32_t* out_col,
              void* out_val, int64_t* nnz, void* stream) {
  SB_TRACE("sb_mm_coo");
  SB_REQUIRE(dtype == SB_F32 || dtype == SB_F64, "sb_mm_coo: dtype must be F32 or F64");
  SB_REQUIRE(h && nnz, "sb_mm_coo: null argument");
  SB_REQUIRE(lower == 0 || lower == 1, "sb_mm_coo: lower must be 0 or 1");
  SB_REQUIRE(h->nentries >= 0 && h->nentries <= kMaxEntries, "sb_mm_coo: bad entry count");
  SB_REQUIRE(h->nentries == 0 || (row && col), "sb_mm_coo: null entries");
  SB_REQUIRE(h->field == SB_MM_PATTERN || h->nentries == 0 || val, "sb_mm_coo: null values");
  SB_REQUIRE(!out_row || (out_col && out_val), "sb_mm_coo: null output");
  int r = ensure_device();
  if (r) return r;
  cudaStream_t st = as_stream(stream);
  if (dtype == SB_F32)
    return mm_coo_impl<float>(lower != 0, h, row, col, val, out_row, out_col, (float*)out_val,
                              nnz, st);
  return mm_coo_impl<double>(lower != 0, h, row, col, val, out_row, out_col, (double*)out_val,
                             nnz, st);
}

}  // extern "C"
