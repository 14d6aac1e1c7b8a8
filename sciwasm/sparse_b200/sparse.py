"""Host mirror of SciWasm.Sparse's JavaScript API over libsparse_b200.so.

The reference module (src/sequential/src/sparse32.js, f64 twin sparse64.js)
keeps matrices as typed arrays in wasm linear memory and exposes
`spmv(A, x, y, inner_max)`, `coo_csr`, `csr_dia`, `csr_ell`, `transpose`,
`eliminate_zeros`, the element-wise maps, `create_vec`, `free`, ...  This
module keeps those names and object shapes (`sparse_COO_t`, `sparse_CSR_t`,
`sparse_DIA_t`, `sparse_ELL_t`, `sparse_vec_t`), but the arrays live in
device memory (HBM) and every operation is a CUDA kernel of
libsparse_b200.so.  There is no CPU compute path.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from ._lib import call

# BF16 value arrays are held as uint16 words (numpy has no bfloat16).
_DT_CODE = {np.dtype(np.float32): _lib.SB_F32, np.dtype(np.float64): _lib.SB_F64,
            np.dtype(np.uint16): _lib.SB_BF16}
_STORAGE = {"f32": np.float32, "f64": np.float64, "bf16": np.uint16}


def _dtcode(dtype) -> int:
    dt = np.dtype(dtype)
    if dt not in _DT_CODE:
        raise TypeError(f"value dtype must be float32, float64 or bf16 (uint16), got {dt}")
    return _DT_CODE[dt]


def _vec_dtype(A):
    """dtype of x and y for matrix A (f32 for BF16-stored values)."""
    return np.dtype(np.float32) if A.dtype == np.uint16 else A.dtype


def _sp(stream) -> Optional[int]:
    return None if stream is None else int(stream)


class DeviceArray:
    """A 1-D array in device memory (the stand-in for a wasm-heap block)."""

    __slots__ = ("n", "dtype", "nbytes", "ptr", "_owned")

    def __init__(self, n: int, dtype, ptr: Optional[int] = None):
        self.ptr, self._owned = 0, False  # a failed allocation leaves nothing to free
        self.n = int(n)
        self.dtype = np.dtype(dtype)
        self.nbytes = self.n * self.dtype.itemsize
        if ptr is None:
            p = C.c_void_p()
            call("sb_malloc", C.byref(p), max(self.nbytes, 16))
            self.ptr = int(p.value)
            self._owned = True
        else:
            self.ptr = int(ptr)
            self._owned = False

    @classmethod
    def from_host(cls, arr, dtype=None, stream=None) -> "DeviceArray":
        a = np.ascontiguousarray(arr, dtype=dtype)
        d = cls(a.size, a.dtype)
        d.upload(a, stream)
        return d

    def upload(self, arr, stream=None) -> None:
        a = np.ascontiguousarray(arr, dtype=self.dtype)
        if a.size != self.n:
            raise ValueError(f"upload of {a.size} elements into an array of {self.n}")
        if self.nbytes:
            call("sb_memcpy_htod", self.ptr, a.ctypes.data, self.nbytes, _sp(stream))
            call("sb_stream_synchronize", _sp(stream))

    def to_host(self, stream=None) -> np.ndarray:
        out = np.empty(self.n, dtype=self.dtype)
        if self.nbytes:
            call("sb_memcpy_dtoh", out.ctypes.data, self.ptr, self.nbytes, _sp(stream))
            call("sb_stream_synchronize", _sp(stream))
        return out

    def fill_zero(self, stream=None) -> None:
        if self.nbytes:
            call("sb_memset", self.ptr, 0, self.nbytes, _sp(stream))

    def free(self) -> None:
        if self._owned and self.ptr:
            try:
                _lib.load().sb_free(self.ptr)
            except Exception:
                pass
        self.ptr = 0
        self._owned = False

    def __del__(self):
        self.free()


class PinnedBuffer:
    """Page-locked host memory (sb_host_alloc) with a numpy byte view, for
    copies that overlap with device work."""

    def __init__(self, nbytes: int):
        self.nbytes = int(nbytes)
        p = C.c_void_p()
        call("sb_host_alloc", C.byref(p), max(self.nbytes, 16))
        self.ptr = int(p.value)
        self.bytes = np.ctypeslib.as_array((C.c_uint8 * max(self.nbytes, 16)).from_address(self.ptr))

    def view(self, offset: int, n: int, dtype) -> np.ndarray:
        dt = np.dtype(dtype)
        return self.bytes[offset:offset + n * dt.itemsize].view(dt)

    def free(self) -> None:
        if self.ptr:
            self.bytes = None
            try:
                _lib.load().sb_host_free(self.ptr)
            except Exception:
                pass
            self.ptr = 0

    def __del__(self):
        self.free()


# --------------------------------------------------------------- objects
# Shapes follow src/sequential/src/sparse32.js:29-198.


class sparse_COO_t:
    """COO matrix: row_index / col_index / val_index arrays of nnz entries.

    rows_sorted is True when row_index is known to be non-decreasing: set by
    coo_from_host (checked on the host) and by the Matrix Market constructors
    (sorted by (row, col)); spmv then adds whole rows without atomics.  Code
    that rewrites row_index in place must reset it."""

    def __init__(self, row_index, col_index, val_index, N, nnz, rows_sorted=False):
        self.row_index, self.col_index, self.val_index = row_index, col_index, val_index
        self.N, self.nnz = int(N), int(nnz)
        self.rows_sorted = bool(rows_sorted)

    @property
    def dtype(self):
        return self.val_index.dtype

    def row_array(self):
        return self.row_index.to_host()

    def col_array(self):
        return self.col_index.to_host()

    def val_array(self):
        return self.val_index.to_host()

    def diagonal(self, offset=0, stream=None):
        """sparse_self_diagonal_coo (src/sequential/src/sparse32.js:314-321):
        the k-th diagonal as a new vector of N - |k| values (None when
        N - |k| <= 0, where the reference returns undefined); rows must be
        sorted, as the reference's COO objects are."""
        k = int(offset)
        count = self.N - (k if k >= 0 else -k)  # (this module's abs is the element-wise map)
        if count <= 0:
            return None
        v = create_vec(count, 0, self.dtype)
        call("sb_diagonal_coo", _dtcode(self.dtype), int(offset), self.row_index.ptr,
             self.col_index.ptr, self.val_index.ptr, v.vec_index.ptr, self.N, self.nnz,
             _sp(stream))
        return v

    def min(self, axis=1, stream=None):
        """sparse_self_min_coo (src/sequential/src/sparse32.js:323-328): per
        row minimum for axis 1 (a zero vector for other axes), with the
        reference's implicit-zero rule and walk."""
        v = create_vec(self.N, 0, self.dtype)
        call("sb_min_coo", _dtcode(self.dtype), int(axis), self.row_index.ptr,
             self.col_index.ptr, self.val_index.ptr, v.vec_index.ptr, self.N, self.nnz,
             _sp(stream))
        return v


def sum_coo(A_coo, axis=1, stream=None):
    """Row sums of a row-sorted COO for axis 1 (sum_coo,
    src/sequential/src/sparse_opt_32.wat:1800-1845), a zero vector otherwise."""
    v = create_vec(A_coo.N, 0, A_coo.dtype)
    call("sb_sum_coo", _dtcode(A_coo.dtype), int(axis), A_coo.row_index.ptr,
         A_coo.col_index.ptr, A_coo.val_index.ptr, v.vec_index.ptr, A_coo.N, A_coo.nnz,
         _sp(stream))
    return v


class sparse_CSC_t:
    """CSC matrix (src/sequential/src/sparse32.js:112-121): col_index (ncols+1
    column pointers), row_index / val_index (nnz)."""

    def __init__(self, col_index, row_index, val_index, ncols, nnz):
        self.col_index, self.row_index, self.val_index = col_index, row_index, val_index
        self.ncols, self.nnz = int(ncols), int(nnz)

    @property
    def dtype(self):
        return self.val_index.dtype

    def col_array(self):
        return self.col_index.to_host()

    def row_array(self):
        return self.row_index.to_host()

    def val_array(self):
        return self.val_index.to_host()


class sparse_CSR_t:
    """CSR matrix: row_index (N+1), col_index / val_index (nnz)."""

    def __init__(self, row_index, col_index, val_index, N, nnz):
        self.row_index, self.col_index, self.val_index = row_index, col_index, val_index
        self.N, self.nnz = int(N), int(nnz)

    @property
    def dtype(self):
        return self.val_index.dtype

    def row_array(self):
        return self.row_index.to_host()

    def col_array(self):
        return self.col_index.to_host()

    def val_array(self):
        return self.val_index.to_host()


class sparse_DIA_t:
    """DIA matrix: offset_index (ndiags), data_index (ndiags*stride), stride N."""

    def __init__(self, offset_index, data_index, ndiags, stride, N, nnz):
        self.offset_index, self.data_index = offset_index, data_index
        self.ndiags, self.stride, self.N, self.nnz = int(ndiags), int(stride), int(N), int(nnz)

    @property
    def dtype(self):
        return self.data_index.dtype

    def offset_array(self):
        return self.offset_index.to_host()

    def data_array(self):
        return self.data_index.to_host()


class sparse_ELL_t:
    """ELL matrix: column-major indices_index / data_index of ncols*N slots."""

    def __init__(self, indices_index, data_index, ncols, N, nnz):
        self.indices_index, self.data_index = indices_index, data_index
        self.ncols, self.N, self.nnz = int(ncols), int(N), int(nnz)

    @property
    def dtype(self):
        return self.data_index.dtype

    def indices_array(self):
        return self.indices_index.to_host()

    def data_array(self):
        return self.data_index.to_host()


class sparse_vec_t:
    """Dense vector of vec_nelem values."""

    def __init__(self, vec_index, vec_nelem):
        self.vec_index = vec_index
        self.vec_nelem = int(vec_nelem)

    @property
    def dtype(self):
        return self.vec_index.dtype

    def array(self):
        return self.vec_index.to_host()

    def size(self):
        return self.vec_nelem


# --------------------------------------------------------------- allocation
# allocate_*: src/sequential/src/sparse32.js:2174-2395.


def allocate_COO(N, nnz, dtype=np.float32):
    return sparse_COO_t(DeviceArray(nnz, np.int32), DeviceArray(nnz, np.int32),
                        DeviceArray(nnz, dtype), N, nnz)


def allocate_CSR(N, nnz, dtype=np.float32):
    return sparse_CSR_t(DeviceArray(N + 1, np.int32), DeviceArray(nnz, np.int32),
                        DeviceArray(nnz, dtype), N, nnz)


def allocate_DIA(N, nnz, ndiags, stride, dtype=np.float32):
    return sparse_DIA_t(DeviceArray(ndiags, np.int32), DeviceArray(ndiags * stride, dtype),
                        ndiags, stride, N, nnz)


def allocate_ELL(N, nnz, ncols, dtype=np.float32):
    return sparse_ELL_t(DeviceArray(ncols * N, np.int32), DeviceArray(ncols * N, dtype),
                        ncols, N, nnz)


def create_vec(nelem, val=0, dtype=np.float32):
    """create_vec (src/sequential/src/sparse32.js:2371-2379)."""
    v = sparse_vec_t(DeviceArray(nelem, dtype), nelem)
    if val == 0:
        v.vec_index.fill_zero()
    else:
        v.vec_index.upload(np.full(nelem, val, dtype=dtype))
    return v


def vec_from_host(arr, dtype=None):
    a = np.ascontiguousarray(arr, dtype=dtype)
    return sparse_vec_t(DeviceArray.from_host(a), a.size)


def _check_indices(name, idx, N):
    if idx.size and (idx.min() < 0 or idx.max() >= N):
        raise ValueError(f"{name} index outside [0, {N})")


def coo_from_host(row, col, val, N, dtype=None):
    """Upload a COO matrix; indices are validated on the host first."""
    row = np.ascontiguousarray(row, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=dtype if dtype is not None else None)
    _dtcode(val.dtype)
    if not (row.size == col.size == val.size):
        raise ValueError("row, col and val must have the same length")
    _check_indices("row", row, N)
    _check_indices("col", col, N)
    return sparse_COO_t(DeviceArray.from_host(row), DeviceArray.from_host(col),
                        DeviceArray.from_host(val), N, row.size,
                        rows_sorted=bool(row.size < 2 or np.all(row[1:] >= row[:-1])))


def csr_from_host(row_ptr, col, val, dtype=None):
    """Upload a CSR matrix after checking row_ptr monotonicity and col range."""
    row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(col, dtype=np.int32)
    val = np.ascontiguousarray(val, dtype=dtype if dtype is not None else None)
    _dtcode(val.dtype)
    N = row_ptr.size - 1
    if N < 0 or row_ptr[0] != 0 or row_ptr[-1] != col.size or col.size != val.size:
        raise ValueError("inconsistent CSR arrays")
    if N and np.any(np.diff(row_ptr) < 0):
        raise ValueError("row_ptr must be non-decreasing")
    _check_indices("col", col, N)
    return sparse_CSR_t(DeviceArray.from_host(row_ptr), DeviceArray.from_host(col),
                        DeviceArray.from_host(val), N, col.size)


def dia_from_host(offset, data, N, nnz=None):
    offset = np.ascontiguousarray(offset, dtype=np.int32)
    data = np.ascontiguousarray(data)
    _dtcode(data.dtype)
    nd = offset.size
    if data.size != nd * N:
        raise ValueError("DIA data must hold ndiags*N values (stride N)")
    if nd and (offset.min() <= -N or offset.max() >= N):
        raise ValueError("DIA offset outside (-N, N)")
    return sparse_DIA_t(DeviceArray.from_host(offset), DeviceArray.from_host(data), nd, N, N,
                        nnz if nnz is not None else int(np.count_nonzero(data)))


def ell_from_host(indices, data, ncols, N, nnz=None):
    indices = np.ascontiguousarray(indices, dtype=np.int32)
    data = np.ascontiguousarray(data)
    _dtcode(data.dtype)
    if indices.size != ncols * N or data.size != ncols * N:
        raise ValueError("ELL arrays must hold ncols*N slots")
    _check_indices("ELL", indices, N)
    return sparse_ELL_t(DeviceArray.from_host(indices), DeviceArray.from_host(data), ncols, N,
                        nnz if nnz is not None else int(np.count_nonzero(data)))


# --------------------------------------------------------------- row reordering


def sort_rows_by_nnz(A_csr, stream=None):
    """sort_rows_by_nnz (src/parallel/src/sparse32.js:2148-2218): a new CSR
    with the rows stably sorted by their number of nonzeros, carrying
    permutation_index (new -> old row), nnz_row_index and num_zero_rows ..
    num_three_rows."""
    N, nnz = A_csr.N, A_csr.nnz
    B = allocate_CSR(N, nnz, A_csr.dtype)
    B.nnz_row_index = DeviceArray(N, np.int32)
    B.permutation_index = DeviceArray(N, np.int32)
    small = (C.c_int32 * 4)()
    call("sb_sort_rows_by_nnz", _dtcode(A_csr.dtype), A_csr.row_index.ptr, A_csr.col_index.ptr,
         A_csr.val_index.ptr, N, nnz, B.row_index.ptr, B.col_index.ptr, B.val_index.ptr,
         B.nnz_row_index.ptr, B.permutation_index.ptr, small, _sp(stream))
    B.num_zero_rows, B.num_one_rows, B.num_two_rows, B.num_three_rows = (int(v) for v in small)
    return B


def reorder_NN(A_csr, w=16, stream=None):
    """reorder_NN (src/parallel/src/sparse32.js:2501-2622): a new CSR whose rows
    follow a greedy nearest-neighbour walk by the Jaccard similarity of their
    16-column cache lines (window of w rows; the reference's callers pass 16
    and the output of sort_rows_by_nnz).  It carries permutation_index (new
    row -> row of the matrix A_csr came from: A_csr's own permutation_index
    composed with the walk, or the walk alone), nnz_row_index (its own row
    lengths; the reference leaves the input order's there) and num_zero_rows ..
    num_three_rows."""
    N, nnz = A_csr.N, A_csr.nnz
    B = allocate_CSR(N, nnz, A_csr.dtype)
    walk = DeviceArray(N, np.int32)
    B.permutation_index = DeviceArray(N, np.int32)
    pin = getattr(A_csr, "permutation_index", None)
    call("sb_reorder_nn", _dtcode(A_csr.dtype), A_csr.row_index.ptr, A_csr.col_index.ptr,
         A_csr.val_index.ptr, N, nnz, int(w), pin.ptr if pin is not None else None, walk.ptr,
         B.permutation_index.ptr, B.row_index.ptr, B.col_index.ptr, B.val_index.ptr,
         _sp(stream))
    lens = np.diff(B.row_array()) if N else np.zeros(0, np.int32)
    B.nnz_row_index = DeviceArray.from_host(lens.astype(np.int32))
    counts = np.bincount(np.minimum(lens, 4), minlength=5)
    B.num_zero_rows = int(counts[0])
    B.num_one_rows = int(counts[:2].sum())
    B.num_two_rows = int(counts[:3].sum())
    B.num_three_rows = int(counts[:4].sum())
    B.walk_index = walk
    return B


def sort_y_rows_by_nnz(y_view, A_csr, stream=None):
    """sort_y_rows_by_nnz (src/parallel/src/sparse32.js:2220-2235): y_view
    (computed with the reordered matrix) back in the original row order; the
    view is given a new array, as the reference replaces y's buffer."""
    N = A_csr.N
    out = DeviceArray(N, y_view.dtype)
    call("sb_unpermute_rows", _dtcode(y_view.dtype), A_csr.permutation_index.ptr,
         y_view.vec_index.ptr, out.ptr, N, _sp(stream))
    y_view.vec_index = out
    return y_view


def calculate_csr_locality_index(A_csr, stream=None) -> float:
    """calculate_csr_locality_index (src/parallel/src/sparse32.js:2238-2269)."""
    v = C.c_double(0.0)
    call("sb_csr_locality_index", A_csr.row_index.ptr, A_csr.col_index.ptr, A_csr.N, A_csr.nnz,
         C.byref(v), _sp(stream))
    return float(v.value)


# --------------------------------------------------------------- Matrix Market


class sparse_MM_info:
    """sparse_MM_info (src/sequential/src/sparse32.js:14-25): the header of a
    Matrix Market file and its entries (1-based, device arrays), with nnz as
    read_matrix_MM_files counts it."""

    _FIELDS = {_lib.SB_MM_REAL: "real", _lib.SB_MM_INTEGER: "integer",
               _lib.SB_MM_PATTERN: "pattern", _lib.SB_MM_COMPLEX: "complex"}

    def __init__(self, header, row, col, val):
        self.header = header
        self.field = self._FIELDS[header.field]
        self.symmetry = "symmetric" if header.symmetric else "general"
        self.nrows, self.ncols, self.nentries = header.nrows, header.ncols, header.nentries
        self.row, self.col, self.val = row, col, val
        self.nnz = self._count(0)

    def _count(self, lower, stream=None):
        n = C.c_int64(0)
        call("sb_mm_coo", _lib.SB_F32, int(lower), C.byref(self.header), self.row.ptr,
             self.col.ptr, self.val.ptr if self.val is not None else None, None, None, None,
             C.byref(n), _sp(stream))
        return int(n.value)


def read_matrix_MM(source, nthreads=0, stream=None) -> sparse_MM_info:
    """read_matrix_MM_files (src/sequential/src/sparse32.js:1956-1981) on a
    file path or the file's bytes: the text is parsed on the host (entry
    lines across nthreads threads), the entries are uploaded to the device."""
    if isinstance(source, (bytes, bytearray, memoryview)):
        text = np.frombuffer(bytes(source), dtype=np.uint8)
    else:
        text = np.fromfile(source, dtype=np.uint8)
    hdr = _lib.MMHeader()
    call("sb_mm_read_header", text.ctypes.data, text.size, C.byref(hdr))
    n = int(hdr.nentries)
    row = np.empty(n, np.int32)
    col = np.empty(n, np.int32)
    pattern = hdr.field == _lib.SB_MM_PATTERN
    val = None if pattern else np.empty(n, np.float64)
    call("sb_mm_read_entries", text.ctypes.data, text.size, C.byref(hdr), row.ctypes.data,
         col.ctypes.data, None if pattern else val.ctypes.data, int(nthreads))
    return sparse_MM_info(hdr, DeviceArray.from_host(row), DeviceArray.from_host(col),
                          None if pattern else DeviceArray.from_host(val))


def _coo_from_mm(mm_info, lower, dtype, stream):
    nnz = mm_info._count(lower, stream)
    A = allocate_COO(mm_info.nrows, nnz, dtype)
    n = C.c_int64(0)
    call("sb_mm_coo", _dtcode(dtype), int(lower), C.byref(mm_info.header), mm_info.row.ptr,
         mm_info.col.ptr, mm_info.val.ptr if mm_info.val is not None else None,
         A.row_index.ptr, A.col_index.ptr, A.val_index.ptr, C.byref(n), _sp(stream))
    A.rows_sorted = True  # sorted by (row, col) on the device
    return A


def create_COO_from_MM(mm_info, dtype=np.float32, stream=None):
    """create_COO_from_MM (src/sequential/src/sparse32.js:2103-2172): a new
    COO with explicit zeros dropped and symmetric entries mirrored, sorted
    by (row, col).  Values in `dtype` (f32 as sparse32.js, f64 as
    sparse64.js)."""
    return _coo_from_mm(mm_info, 0, dtype, stream)


def create_LCOO_from_MM(mm_info, dtype=np.float32, stream=None):
    """create_LCOO_from_MM (src/sequential/src/sparse32.js:1983-2099): the
    strictly lower triangle (symmetric upper entries mirrored, zeros
    dropped) plus a unit diagonal, sorted by (row, col) so that each row's
    diagonal is its last entry."""
    return _coo_from_mm(mm_info, 1, dtype, stream)


def mmread(filename, dtype=np.float32, nthreads=0):
    """mmread (src/sequential/src/sparse32.js:2499-2510): read a Matrix
    Market file into a new device COO."""
    return create_COO_from_MM(read_matrix_MM(filename, nthreads), dtype)


def free(obj) -> None:
    """free (src/sequential/src/sparse32.js:2204-2231)."""
    if obj is None:
        return
    for name in ("row_index", "col_index", "val_index", "offset_index", "data_index",
                 "indices_index", "vec_index"):
        arr = getattr(obj, name, None)
        if isinstance(arr, DeviceArray):
            arr.free()


# --------------------------------------------------------------- SpMV


def csr_autotune(A_csr, x_view, reps=5, stream=None):
    """Pick the fastest CSR kernel options for this matrix (timed on a scratch
    y; the choice is cached on the object and used by spmv)."""
    best = _lib.CsrOpts()
    ms = C.c_float(0)
    call("sb_csr_autotune", _dtcode(A_csr.dtype), A_csr.row_index.ptr, A_csr.col_index.ptr,
         A_csr.val_index.ptr, x_view.vec_index.ptr, A_csr.N, A_csr.nnz, int(reps), C.byref(best),
         C.byref(ms), _sp(stream))
    A_csr.opts = best
    return {"kernel": best.kernel, "lanes_per_row": best.lanes_per_row, "unroll": best.unroll,
            "grid": best.grid, "ms": float(ms.value)}


def csr_coo(A_csr, stream=None):
    """The COO form of a CSR matrix (rows expanded from row_ptr, so
    rows_sorted holds); no counterpart in the reference."""
    B = allocate_COO(A_csr.N, A_csr.nnz, A_csr.dtype)
    call("sb_csr_coo", _dtcode(A_csr.dtype), A_csr.row_index.ptr, A_csr.col_index.ptr,
         A_csr.val_index.ptr, A_csr.N, A_csr.nnz, B.row_index.ptr, B.col_index.ptr,
         B.val_index.ptr, _sp(stream))
    B.rows_sorted = True
    return B


_FORMAT_NAMES = ("csr", "dia", "ell", "coo")


def spmv_autotune(A_csr, x_view=None, reps=5, timed=True, stream=None):
    """Choose the SpMV format and kernel for a CSR matrix (sb_spmv_autotune):
    the reference's admission test and the compulsory bytes of each format
    decide what is tried; with timed=True device timing decides among them,
    with timed=False the statistics alone (fewest bytes; x_view unused).
    Returns (M, info): M is the matrix in the chosen format -- A_csr itself,
    with its CSR kernel options set, when CSR wins; a new DIA, ELL or COO
    object built on the device otherwise -- and info holds the statistics,
    bytes and per-format times."""
    ch = _lib.SpmvChoice()
    if timed and x_view is None:
        raise ValueError("spmv_autotune: the timed mode needs an x vector")
    call("sb_spmv_autotune", _dtcode(A_csr.dtype), A_csr.row_index.ptr, A_csr.col_index.ptr,
         A_csr.val_index.ptr, x_view.vec_index.ptr if x_view is not None else None, A_csr.N,
         A_csr.nnz, _lib.SB_TUNE_TIMED if timed else _lib.SB_TUNE_MODEL, int(reps),
         C.byref(ch), _sp(stream))
    A_csr.opts = _lib.CsrOpts(ch.csr.kernel, ch.csr.lanes_per_row, ch.csr.unroll, ch.csr.grid)
    fmt = _FORMAT_NAMES[ch.format]
    if fmt == "dia":
        M = csr_dia(A_csr, stream)
    elif fmt == "ell":
        M = csr_ell(A_csr, stream)
    elif fmt == "coo":
        M = csr_coo(A_csr, stream)
    else:
        M = A_csr
    info = {"format": fmt,
            "csr_opts": {"kernel": ch.csr.kernel, "lanes_per_row": ch.csr.lanes_per_row,
                         "unroll": ch.csr.unroll, "grid": ch.csr.grid},
            "ndiags": ch.ndiags, "ncols": ch.ncols, "dia_admitted": bool(ch.dia_admitted),
            "ell_admitted": bool(ch.ell_admitted),
            "ms": {n: (round(float(ch.ms[k]), 4) if ch.ms[k] >= 0 else None)
                   for k, n in enumerate(_FORMAT_NAMES)},
            "bytes": {n: int(ch.bytes[k]) for k, n in enumerate(_FORMAT_NAMES)}}
    return M, info


def spmv(A, x_view, y_view, inner_max=1, stream=None):
    """y <- y + A x, inner_max times (src/sequential/src/sparse32.js:1232-1286).

    Returns None like the reference; raises for an undefined matrix instead of
    logging (the reference prints "spmv input : undefined" and returns)."""
    if A is None:
        raise ValueError("spmv input : undefined")
    if x_view.dtype != _vec_dtype(A) or y_view.dtype != _vec_dtype(A):
        raise TypeError("x and y must have the matrix's value dtype (f32 for BF16 storage)")
    if A.dtype == np.uint16 and not isinstance(A, (sparse_CSR_t, sparse_DIA_t)):
        raise TypeError("BF16 storage is supported for CSR and DIA SpMV")
    if x_view.vec_nelem < A.N or y_view.vec_nelem < A.N:
        raise ValueError("x and y must hold N values")
    dt = _dtcode(A.dtype)
    s = _sp(stream)
    x, y = x_view.vec_index.ptr, y_view.vec_index.ptr
    if isinstance(A, sparse_COO_t):
        flags = _lib.SB_COO_ROWS_SORTED if getattr(A, "rows_sorted", False) else 0
        call("sb_spmv_coo_ex", dt, A.row_index.ptr, A.col_index.ptr, A.val_index.ptr, x, y, A.N,
             A.nnz, inner_max, flags, s)
    elif isinstance(A, sparse_CSR_t):
        opts = getattr(A, "opts", None)
        if opts is None:
            call("sb_spmv_csr", dt, A.row_index.ptr, A.col_index.ptr, A.val_index.ptr, x, y, A.N,
                 A.nnz, inner_max, s)
        else:
            call("sb_spmv_csr_ex", dt, A.row_index.ptr, A.col_index.ptr, A.val_index.ptr, x, y,
                 A.N, A.nnz, inner_max, C.byref(opts), s)
    elif isinstance(A, sparse_DIA_t):
        call("sb_spmv_dia", dt, A.offset_index.ptr, A.data_index.ptr, A.N, A.ndiags, A.stride, x,
             y, inner_max, s)
    elif isinstance(A, sparse_ELL_t):
        call("sb_spmv_ell", dt, A.indices_index.ptr, A.data_index.ptr, A.N, A.ncols, x, y,
             inner_max, s)
    else:
        raise TypeError(f"spmv: unsupported matrix object {type(A).__name__}")


def convert_values(src, storage, stream=None):
    """A new device array holding src's values in `storage` ("f32", "f64",
    "bf16"), rounded to nearest even."""
    out = DeviceArray(src.n, _STORAGE[storage])
    call("sb_convert_values", _dtcode(src.dtype), src.ptr, _dtcode(out.dtype), out.ptr, src.n,
         _sp(stream))
    return out


def csr_with_storage(A_csr, storage, stream=None):
    """The same CSR structure with values stored as `storage` (shares
    row_index/col_index with A_csr)."""
    return sparse_CSR_t(A_csr.row_index, A_csr.col_index,
                        convert_values(A_csr.val_index, storage, stream), A_csr.N, A_csr.nnz)


def with_storage(A, storage, stream=None):
    """A CSR, DIA or ELL matrix with its values stored as `storage` (the
    index arrays are shared with A).  BF16 values serve the batched SpMV
    (f32 vectors and sums); the single-call DIA and ELL kernels take f32 and
    f64 only."""
    if isinstance(A, sparse_CSR_t):
        return csr_with_storage(A, storage, stream)
    if isinstance(A, sparse_DIA_t):
        return sparse_DIA_t(A.offset_index, convert_values(A.data_index, storage, stream),
                            A.ndiags, A.stride, A.N, A.nnz)
    if isinstance(A, sparse_ELL_t):
        return sparse_ELL_t(A.indices_index, convert_values(A.data_index, storage, stream),
                            A.ncols, A.N, A.nnz)
    raise TypeError(f"with_storage: {type(A).__name__} is not CSR, DIA or ELL")


# --------------------------------------------------------------- batched SpMV


class BatchExecutor:
    """Batched SpMV over many matrices (CSR, DIA or ELL, values stored as
    `storage`) and right-hand sides in one graph-replayed persistent launch."""

    def __init__(self, storage="f32", capacity=1024):
        self.storage = storage
        self.capacity = int(capacity)
        p = C.c_void_p()
        call("sb_batch_exec_create", _dtcode(_STORAGE[storage]), self.capacity, C.byref(p))
        self.ptr = p.value
        self._items = (_lib.BatchItem * self.capacity)()
        self._keep = []

    def run(self, jobs, stream=None, overwrite=False, lanes=0):
        """jobs: iterable of (A, x DeviceArray N*k, y DeviceArray N*k, k) with A
        a CSR, DIA (stride N) or ELL matrix; y += A x, or y = A x with
        overwrite=True.  lanes: lanes per CSR row for every item (0 = chosen
        per matrix from its mean row length; see sb_batch_item)."""
        self.launch(self.prepare(jobs, overwrite, lanes), stream)

    def prepare(self, jobs, overwrite=False, lanes=0) -> int:
        """Fill the item descriptors for `jobs` (as run) without launching;
        returns the item count for launch().  The descriptors stay valid until
        the next prepare(), so a fixed batch is prepared once and launched
        many times."""
        jobs = list(jobs)
        if len(jobs) > self.capacity:
            raise ValueError(f"{len(jobs)} items exceed the executor capacity {self.capacity}")
        n = 0
        self._keep = []
        for A, x, y, k in jobs:
            it = self._items[n]
            it.x, it.y = x.ptr, y.ptr
            it.N, it.nrhs, it.lanes, it.nnz = A.N, int(k), int(lanes), A.nnz
            it.flags = 1 if overwrite else 0
            if isinstance(A, sparse_DIA_t):
                if A.stride != A.N:
                    raise ValueError("batched DIA items need stride == N")
                it.row_ptr, it.col, it.val = A.offset_index.ptr, None, A.data_index.ptr
                it.format, it.width = _lib.SB_FMT_DIA, A.ndiags
            elif isinstance(A, sparse_ELL_t):
                it.row_ptr, it.col, it.val = None, A.indices_index.ptr, A.data_index.ptr
                it.format, it.width = _lib.SB_FMT_ELL, A.ncols
            else:
                it.row_ptr, it.col, it.val = A.row_index.ptr, A.col_index.ptr, A.val_index.ptr
                it.format, it.width = _lib.SB_FMT_CSR, 0
            self._keep.append((A, x, y))
            n += 1
        return n

    def launch(self, n, stream=None):
        """Run the batch that prepare() described (its first n items)."""
        call("sb_batch_exec_run", self.ptr, self._items, int(n), _sp(stream))

    def close(self):
        if getattr(self, "ptr", None):
            try:
                _lib.load().sb_batch_exec_destroy(self.ptr)
            except Exception:
                pass
            self.ptr = None

    def __del__(self):
        self.close()


# --------------------------------------------------------------- conversions


def coo_csr(A_coo, stream=None):
    """coo_csr (src/sequential/src/sparse32.js:1674-1720): a new CSR object,
    entries stably ordered by (row, col) exactly as the reference's count /
    scan / scatter / per-row stable sort produces them."""
    A = allocate_CSR(A_coo.N, A_coo.nnz, A_coo.dtype)
    call("sb_coo_csr", _dtcode(A_coo.dtype), A_coo.row_index.ptr, A_coo.col_index.ptr,
         A_coo.val_index.ptr, A_coo.N, A_coo.nnz, A.row_index.ptr, A.col_index.ptr,
         A.val_index.ptr, _sp(stream))
    return A


def coo_csc(A_coo, stream=None):
    """coo_csc (src/sequential/src/sparse32.js:1629-1671): a new CSC, entries
    stably ordered by (col, row)."""
    N, nnz = A_coo.N, A_coo.nnz
    B = sparse_CSC_t(DeviceArray(N + 1, np.int32), DeviceArray(nnz, np.int32),
                     DeviceArray(nnz, A_coo.dtype), N, nnz)
    call("sb_coo_csc", _dtcode(A_coo.dtype), A_coo.row_index.ptr, A_coo.col_index.ptr,
         A_coo.val_index.ptr, N, nnz, B.col_index.ptr, B.row_index.ptr, B.val_index.ptr,
         _sp(stream))
    return B


def spts_csc(A_csc, x_view, y_view, stream=None):
    """spts_csc (src/sequential/src/sparse_opt_32.wat:11-148): solve L y = x
    for a CSC lower triangle whose columns start with their diagonal."""
    if x_view.dtype != A_csc.dtype or y_view.dtype != A_csc.dtype:
        raise TypeError("x, y and the matrix must share one value dtype")
    call("sb_spts_csc", _dtcode(A_csc.dtype), A_csc.col_index.ptr, A_csc.row_index.ptr,
         A_csc.val_index.ptr, A_csc.ncols, A_csc.nnz, x_view.vec_index.ptr,
         y_view.vec_index.ptr, _sp(stream))


def num_cols(A_csr, stream=None) -> int:
    """num_cols (src/sequential/src/sparse32.js:1436-1447)."""
    nc = C.c_int32(0)
    call("sb_num_cols", A_csr.row_index.ptr, A_csr.N, C.byref(nc), _sp(stream))
    return int(nc.value)


def csr_ell(A_csr, stream=None):
    """csr_ell (src/sequential/src/sparse32.js:1449-1484).  Returns None when
    the reference's admission test refuses (it logs and returns undefined)."""
    nc = num_cols(A_csr, stream)
    lib = _lib.load()
    if not lib.sb_ell_admitted(nc, A_csr.N, A_csr.nnz):
        return None
    E = allocate_ELL(A_csr.N, A_csr.nnz, nc, A_csr.dtype)
    call("sb_csr_ell", _dtcode(A_csr.dtype), A_csr.row_index.ptr, A_csr.col_index.ptr,
         A_csr.val_index.ptr, A_csr.N, A_csr.nnz, nc, E.indices_index.ptr, E.data_index.ptr,
         _sp(stream))
    return E


def num_diags(A_csr, stream=None):
    """num_diags (src/sequential/src/sparse32.js:1486-1512): [nd, stride]."""
    nd = C.c_int32(0)
    stride = C.c_int32(0)
    call("sb_num_diags", A_csr.row_index.ptr, A_csr.col_index.ptr, A_csr.N, C.byref(nd),
         C.byref(stride), _sp(stream))
    return [int(nd.value), int(stride.value)]


def csr_dia(A_csr, stream=None):
    """csr_dia (src/sequential/src/sparse32.js:1515-1574).  Returns None when
    the admission test refuses."""
    nd, stride = num_diags(A_csr, stream)
    lib = _lib.load()
    if not lib.sb_dia_admitted(nd, stride, A_csr.nnz):
        return None
    D = allocate_DIA(A_csr.N, A_csr.nnz, nd, stride, A_csr.dtype)
    call("sb_csr_dia", _dtcode(A_csr.dtype), A_csr.row_index.ptr, A_csr.col_index.ptr,
         A_csr.val_index.ptr, A_csr.N, A_csr.nnz, nd, stride, D.offset_index.ptr,
         D.data_index.ptr, _sp(stream))
    return D


# --------------------------------------------------------------- transpose / eliminate_zeros


def _d(arr):
    return arr.ptr


def transpose(A, stream=None):
    """transpose (src/sequential/src/sparse32.js:1106-1138): a new object."""
    dt, sp = _dtcode(A.dtype), _sp(stream)
    if isinstance(A, sparse_COO_t):
        B = allocate_COO(A.N, A.nnz, A.dtype)
        call("sb_transpose_coo", dt, _d(A.row_index), _d(A.col_index), _d(A.val_index), A.nnz,
             _d(B.row_index), _d(B.col_index), _d(B.val_index), sp)
        return B
    if isinstance(A, sparse_CSR_t):
        B = allocate_CSR(A.N, A.nnz, A.dtype)
        call("sb_transpose_csr", dt, _d(A.row_index), _d(A.col_index), _d(A.val_index), A.N,
             A.nnz, _d(B.row_index), _d(B.col_index), _d(B.val_index), sp)
        return B
    if isinstance(A, sparse_DIA_t):
        B = allocate_DIA(A.N, A.nnz, A.ndiags, A.stride, A.dtype)
        call("sb_transpose_dia", dt, _d(A.offset_index), _d(A.data_index), A.ndiags, A.stride,
             A.N, _d(B.offset_index), _d(B.data_index), sp)
        return B
    if isinstance(A, sparse_ELL_t):
        cc = C.c_int32(0)
        call("sb_count_transpose_cols_ell", dt, _d(A.data_index), _d(A.indices_index), A.ncols,
             A.N, C.byref(cc), sp)
        B = allocate_ELL(A.N, A.nnz, int(cc.value), A.dtype)
        call("sb_transpose_ell", dt, _d(A.data_index), _d(A.indices_index), A.ncols, A.N,
             B.ncols, _d(B.data_index), _d(B.indices_index), sp)
        return B
    raise TypeError(f"transpose: unsupported object {type(A).__name__}")


def _copy_arrays(pairs, stream):
    for src, dst in pairs:
        call("sb_memcpy_dtod", dst.ptr, src.ptr, src.nbytes, _sp(stream))


def eliminate_zeros(A, stream=None):
    """eliminate_zeros (src/sequential/src/sparse32.js:1140-1207): a new object
    without entries whose value is not (v > 0 || v < 0); an unchanged copy
    when the nonzero count equals A.nnz."""
    dt, sp = _dtcode(A.dtype), _sp(stream)
    if isinstance(A, (sparse_COO_t, sparse_CSR_t)):
        cnt = C.c_int64(0)
        call("sb_count_nonzeros", dt, _d(A.val_index), A.nnz, C.byref(cnt), sp)
        count = int(cnt.value)
        if isinstance(A, sparse_COO_t):
            B = allocate_COO(A.N, A.nnz if count == A.nnz else count, A.dtype)
            if count == A.nnz:
                _copy_arrays([(A.row_index, B.row_index), (A.col_index, B.col_index),
                              (A.val_index, B.val_index)], stream)
            else:
                call("sb_copy_nonzeros_coo", dt, _d(A.row_index), _d(A.col_index),
                     _d(A.val_index), A.nnz, _d(B.row_index), _d(B.col_index),
                     _d(B.val_index), sp)
            B.rows_sorted = A.rows_sorted  # the kept entries stay in order
            return B
        B = allocate_CSR(A.N, A.nnz if count == A.nnz else count, A.dtype)
        if count == A.nnz:
            _copy_arrays([(A.row_index, B.row_index), (A.col_index, B.col_index),
                          (A.val_index, B.val_index)], stream)
        else:
            call("sb_copy_nonzeros_csr", dt, _d(A.row_index), _d(A.col_index), _d(A.val_index),
                 A.N, A.nnz, _d(B.row_index), _d(B.col_index), _d(B.val_index), sp)
        return B
    if isinstance(A, sparse_DIA_t):
        cd = C.c_int32(0)
        cnt = C.c_int64(0)
        call("sb_count_nonzeros_dia", dt, _d(A.offset_index), _d(A.data_index), A.ndiags,
             A.stride, A.N, C.byref(cd), C.byref(cnt), sp)
        if int(cnt.value) == A.nnz:
            B = allocate_DIA(A.N, A.nnz, A.ndiags, A.stride, A.dtype)
            _copy_arrays([(A.offset_index, B.offset_index), (A.data_index, B.data_index)], stream)
            return B
        B = allocate_DIA(A.N, int(cnt.value), int(cd.value), A.stride, A.dtype)
        call("sb_copy_nonzeros_dia", dt, _d(A.offset_index), _d(A.data_index), A.ndiags, A.stride,
             A.N, _d(B.offset_index), _d(B.data_index), sp)
        return B
    if isinstance(A, sparse_ELL_t):
        cc = C.c_int32(0)
        cnt = C.c_int64(0)
        call("sb_count_nonzeros_ell", dt, _d(A.data_index), A.ncols, A.N, C.byref(cc),
             C.byref(cnt), sp)
        if int(cnt.value) == A.nnz:
            B = allocate_ELL(A.N, A.nnz, A.ncols, A.dtype)
            _copy_arrays([(A.indices_index, B.indices_index), (A.data_index, B.data_index)],
                         stream)
            return B
        B = allocate_ELL(A.N, int(cnt.value), int(cc.value), A.dtype)
        call("sb_copy_nonzeros_ell", dt, _d(A.data_index), _d(A.indices_index), A.ncols, A.N,
             B.ncols, _d(B.data_index), _d(B.indices_index), sp)
        return B
    raise TypeError(f"eliminate_zeros: unsupported object {type(A).__name__}")


# --------------------------------------------------------------- element-wise maps
# Functional forms (src/sequential/src/sparse32.js:671-1104) return a copy;
# map_inplace is the self_* method form (:202-667).

MAP_OPS = {"expm1": 0, "log1p": 1, "sin": 2, "tan": 3, "pow": 4, "deg2rad": 5, "rad2deg": 6,
           "sign": 7, "abs": 8, "neg": 9, "sqrt": 10, "ceil": 11, "floor": 12, "trunc": 13,
           "nearest": 14, "multiply": 15}


def _map_into(A, B, op, p, stream):
    dt, sp = _dtcode(A.dtype), _sp(stream)
    code = MAP_OPS[op]
    if isinstance(A, (sparse_COO_t, sparse_CSR_t)):
        call("sb_map_coo", dt, code, float(p), _d(A.val_index), _d(B.val_index), A.nnz, sp)
    elif isinstance(A, sparse_DIA_t):
        call("sb_map_dia", dt, code, float(p), _d(A.offset_index), _d(A.data_index),
             _d(B.data_index), A.ndiags, A.stride, A.N, sp)
    elif isinstance(A, sparse_ELL_t):
        call("sb_map_ell", dt, code, float(p), _d(A.data_index), _d(B.data_index), A.ncols, A.N,
             sp)
    else:
        raise TypeError(f"{op}: unsupported object {type(A).__name__}")


def _copy_structure(A, stream):
    if isinstance(A, sparse_COO_t):
        B = allocate_COO(A.N, A.nnz, A.dtype)
        _copy_arrays([(A.row_index, B.row_index), (A.col_index, B.col_index)], stream)
        B.rows_sorted = A.rows_sorted
    elif isinstance(A, sparse_CSR_t):
        B = allocate_CSR(A.N, A.nnz, A.dtype)
        _copy_arrays([(A.row_index, B.row_index), (A.col_index, B.col_index)], stream)
    elif isinstance(A, sparse_DIA_t):
        B = allocate_DIA(A.N, A.nnz, A.ndiags, A.stride, A.dtype)
        _copy_arrays([(A.offset_index, B.offset_index)], stream)
    elif isinstance(A, sparse_ELL_t):
        B = allocate_ELL(A.N, A.nnz, A.ncols, A.dtype)
        _copy_arrays([(A.indices_index, B.indices_index)], stream)
    else:
        raise TypeError(type(A).__name__)
    return B


def map_copy(A, op, p=0.0, stream=None):
    B = _copy_structure(A, stream)
    _map_into(A, B, op, p, stream)
    return B


def map_inplace(A, op, p=0.0, stream=None):
    _map_into(A, A, op, p, stream)


def expm1(A): return map_copy(A, "expm1")
def log1p(A): return map_copy(A, "log1p")
def sin(A): return map_copy(A, "sin")
def tan(A): return map_copy(A, "tan")
def pow(A, p): return map_copy(A, "pow", p)  # noqa: A001
def deg2rad(A): return map_copy(A, "deg2rad", np.pi)
def rad2deg(A): return map_copy(A, "rad2deg", np.pi)
def sign(A): return map_copy(A, "sign")
def abs(A): return map_copy(A, "abs")  # noqa: A001
def neg(A): return map_copy(A, "neg")
def sqrt(A): return map_copy(A, "sqrt")
def ceil(A): return map_copy(A, "ceil")
def floor(A): return map_copy(A, "floor")
def trunc(A): return map_copy(A, "trunc")
def nearest(A): return map_copy(A, "nearest")
def multiply(A, s): return map_copy(A, "multiply", s)


# --------------------------------------------------------------- level sets / SpTS

_SPTS_ALGO = {"level": _lib.SB_SPTS_LEVEL, "syncfree": _lib.SB_SPTS_SYNCFREE,
              "hybrid": _lib.SB_SPTS_HYBRID}
_SPTS_POLICY = {"native": _lib.SB_SPTS_ACC_NATIVE, "f64": _lib.SB_SPTS_ACC_F64}


class SptsPlan:
    """Level-set analysis of a CSR matrix (owns the device plan; keeps the
    analysed matrix alive because the sync-free solve reads it)."""

    def __init__(self, A_csr, stream=None):
        self.A = A_csr
        p = C.c_void_p()
        call("sb_spts_analyze", _dtcode(A_csr.dtype), A_csr.row_index.ptr, A_csr.col_index.ptr,
             A_csr.val_index.ptr, A_csr.N, A_csr.nnz, _sp(stream), C.byref(p))
        self.ptr = p.value
        nl = C.c_int32(0)
        ok = C.c_int32(0)
        call("sb_spts_plan_info", self.ptr, C.byref(nl), C.byref(ok))
        self.nlevels = int(nl.value)
        self.solvable = bool(ok.value)
        ms = C.c_float(0.0)
        call("sb_spts_plan_analysis_ms", self.ptr, C.byref(ms))
        self.analysis_ms = float(ms.value)

    def levels(self, stream=None):
        """(level, level_ptr, permutation, order) as device arrays."""
        N = self.A.N
        lv, perm, order = (DeviceArray(N, np.int32) for _ in range(3))
        lp = DeviceArray(self.nlevels + 1, np.int32)
        call("sb_spts_plan_levels", self.ptr, lv.ptr, lp.ptr, perm.ptr, order.ptr, _sp(stream))
        call("sb_stream_synchronize", _sp(stream))
        return lv, lp, perm, order

    def growth(self, stream=None) -> float:
        """max_i sum_{j<i} |L_ij| / |L_ii| (below 1: row diagonally dominant)."""
        g = C.c_double(0.0)
        call("sb_spts_plan_growth", self.ptr, C.byref(g), _sp(stream))
        return float(g.value)

    def close(self):
        if getattr(self, "ptr", None):
            try:
                _lib.load().sb_spts_plan_destroy(self.ptr)
            except Exception:
                pass
            self.ptr = None

    def __del__(self):
        self.close()


class SptsBatch:
    """Many triangular solves, each on its own SptsPlan, in one graph-replayed
    persistent launch; every result is bit-identical to
    spts(L, b, y, algo="hybrid", policy=policy)."""

    def __init__(self, dtype=np.float32, policy="native", capacity=256, blocks_per_sm=0):
        """blocks_per_sm > 0 caps the launch at that many blocks per SM, whose
        warps take chunks until the batch is done (sb_spts_batch_set_grid)."""
        self.dtype = np.dtype(dtype)
        self.policy = policy
        self.capacity = int(capacity)
        p = C.c_void_p()
        call("sb_spts_batch_create", _dtcode(self.dtype), _SPTS_POLICY[policy], self.capacity,
             C.byref(p))
        self.ptr = p.value
        if blocks_per_sm:
            call("sb_spts_batch_set_grid", self.ptr, int(blocks_per_sm))
        self._items = (_lib.SptsBatchItem * self.capacity)()
        self._keep = []

    def run(self, jobs, stream=None):
        """jobs: iterable of (SptsPlan, b DeviceArray, y DeviceArray[, work
        DeviceArray]), natural order.  With a work vector (N values of the
        plan's dtype) a solve does not use its plan's own, so a plan may
        repeat in one run and run beside other solves of it."""
        jobs = list(jobs)
        if len(jobs) > self.capacity:
            raise ValueError(f"{len(jobs)} solves exceed the executor capacity {self.capacity}")
        n = 0
        self._keep = []
        for job in jobs:
            plan, b, y = job[:3]
            work = job[3] if len(job) > 3 else None
            it = self._items[n]
            it.plan, it.b, it.y = plan.ptr, b.ptr, y.ptr
            it.work = work.ptr if work is not None else None
            self._keep.append(job)
            n += 1
        call("sb_spts_batch_run", self.ptr, self._items, n, _sp(stream))

    def close(self):
        if getattr(self, "ptr", None):
            try:
                _lib.load().sb_spts_batch_destroy(self.ptr)
            except Exception:
                pass
            self.ptr = None

    def __del__(self):
        self.close()


def CSR_create_level_sets(A_csr, stream=None):
    """CSR_create_level_sets (src/parallel/src/sparse32.js:2942-3008): attaches
    nlevels, level_index (level_ptr) and permutation_index to A_csr."""
    plan = SptsPlan(A_csr, stream)
    lv, lp, perm, order = plan.levels(stream)
    A_csr.nlevels, A_csr.level_index, A_csr.permutation_index = plan.nlevels, lp, perm
    A_csr.level_per_row, A_csr.order_index, A_csr._plan = lv, order, plan
    return A_csr


def CSR_create_level_sets_with_reorder(A_csr, stream=None):
    """CSR_create_level_sets_with_reorder (src/parallel/src/sparse32.js:3010-3181):
    a new CSR whose rows are ordered by level and whose columns are relabelled
    by order[], carrying nlevels, level_index, permutation_index."""
    plan = SptsPlan(A_csr, stream)
    lv, lp, perm, order = plan.levels(stream)
    R = allocate_CSR(A_csr.N, A_csr.nnz, A_csr.dtype)
    call("sb_spts_plan_reordered", plan.ptr, R.row_index.ptr, R.col_index.ptr, R.val_index.ptr,
         _sp(stream))
    call("sb_stream_synchronize", _sp(stream))
    R.nlevels, R.level_index, R.permutation_index = plan.nlevels, lp, perm
    R.level_per_row, R.order_index, R._plan = lv, order, plan
    return R


def _device_status() -> int:
    code = C.c_int(0)
    call("sb_device_status", C.byref(code))
    return int(code.value)


def spts(L, b_view, y_view, algo="level", policy="native", stream=None, check=True):
    """Solve L y = b for a lower-triangular CSR L with its diagonal stored last
    in every row (b, y in natural row order).  algo: "level" (level by level),
    "syncfree" (ready flags, natural order) or "hybrid" (ready flags, level
    order).  policy "f64" accumulates and divides in f64 for f32 values."""
    plan = getattr(L, "_plan", None)
    if plan is None or plan.ptr is None:
        plan = SptsPlan(L, stream)
        L._plan = plan
    if b_view.dtype != L.dtype or y_view.dtype != L.dtype:
        raise TypeError("b, y and L must share one value dtype")
    call("sb_spts_solve", plan.ptr, _SPTS_ALGO[algo], _SPTS_POLICY[policy], b_view.vec_index.ptr,
         y_view.vec_index.ptr, _sp(stream))
    if check:
        call("sb_stream_synchronize", _sp(stream))
        st = _device_status()
        if st:
            raise _lib.SparseError("sb_spts_solve", _lib.SB_ETIMEOUT,
                                   f"device status {st}: a dependency wait ran out")


def spts_csr_sync_free(L, b_view, y_view, spin_limit_cycles=0, stream=None):
    """The raw sync-free kernel (src/parallel/src/spts_opt_32.wat:8-260) on the
    caller's arrays, without structural checks; waits are bounded."""
    call("sb_spts_syncfree_csr", _dtcode(L.dtype), L.row_index.ptr, L.col_index.ptr,
         L.val_index.ptr, L.N, b_view.vec_index.ptr, y_view.vec_index.ptr,
         int(spin_limit_cycles), _sp(stream))


def synchronize(stream=None) -> None:
    call("sb_stream_synchronize", _sp(stream))


# --------------------------------------------------------------- partitioning


def static_nnz(row_ptr, num_workers):
    """static_nnz (src/parallel/src/sparse32.js:2769-2821) on host row
    pointers: greedy contiguous row ranges, each taking rows while its running
    nonzero count is below floor(remaining nnz / remaining workers); the last
    range always ends at N.  Returns (row_start, row_end) int32 arrays.  Used
    here to shard a matrix's rows across GPUs."""
    rp = np.asarray(row_ptr, dtype=np.int64)
    N = rp.size - 1
    nw = int(num_workers)
    rs = np.zeros(nw, np.int32)
    re = np.zeros(nw, np.int32)
    lens = np.diff(rp)
    rem_nnz = int(rp[-1] - rp[0])
    rem_nw = nw
    index = 0
    i = 0
    for i in range(nw):
        if index == N:
            rs[i] = re[i] = N
            continue
        ideal = rem_nnz // rem_nw
        rs[i] = index
        # rows are taken while the running sum is below `ideal`: find the
        # first prefix whose sum reaches it (the reference's loop, vectorised)
        csum = np.cumsum(lens[index:])
        k = int(np.searchsorted(csum, ideal, side="left")) if ideal > 0 else -1
        taken = min(k + 1, N - index) if ideal > 0 else 0
        s = int(csum[taken - 1]) if taken > 0 else 0
        index += taken
        if index < N:
            re[i] = index
        rem_nnz -= s
        rem_nw -= 1
    re[i] = N
    return rs, re


# --------------------------------------------------------------- checksum


def fletcher_sum(a) -> int:
    """fletcher_sum (src/sequential/src/sparse32.js:1291-1304) on host values:
    sum1 = (sum1 + a_i) mod 255, sum2 = (sum2 + sum1) mod 255 with a floored
    modulo on doubles; result parseInt(sum2*256 + sum1)."""
    s1 = 0.0
    s2 = 0.0
    for v in np.asarray(a, dtype=np.float64).tolist():
        t = s1 + v
        s1 = t - np.floor(t / 255.0) * 255.0
        t = s2 + s1
        s2 = t - np.floor(t / 255.0) * 255.0
    return int(s2 * 256.0 + s1)


def clear_vec(y_view, stream=None) -> None:
    """clear_vec (src/sequential/src/sparse32.js:1319-1322): y = 0, on the
    device (stream-ordered).  The reference's benchmark clears y this way
    before every spmv (src/sequential/tests/main32.js:123-124)."""
    y_view.vec_index.fill_zero(stream)


def init_x(x_view) -> None:
    """init_x (src/sequential/src/sparse32.js:1313-1317): x[i] = i."""
    x_view.vec_index.upload(np.arange(x_view.vec_nelem, dtype=x_view.dtype))


def fletcher_sum_y(y_view) -> int:
    """fletcher_sum_y (src/sequential/src/sparse32.js:1306-1311)."""
    return fletcher_sum(y_view.array())
