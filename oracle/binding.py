"""ctypes binding of the CPU oracle (liboracle_sparse.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, as the checker and the timed CPU baseline.  The
product package never imports this module.  Parity status of the oracle:
pinned to the reference's WebAssembly kernels and JavaScript functions by
vectors executed from their source (see sparse_oracle.h).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_sparse.so")

_P = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64

_SIG = {
    "or_spmv_coo_f32": ([_P, _P, _P, _P, _P, _I64], None),
    "or_spmv_coo_f64": ([_P, _P, _P, _P, _P, _I64], None),
    "or_spmv_csr_f32": ([_P, _P, _P, _P, _P, _I32], None),
    "or_spmv_csr_f64": ([_P, _P, _P, _P, _P, _I32], None),
    "or_spmv_dia_f32": ([_P, _P, _I32, _I32, _I32, _P, _P], None),
    "or_spmv_dia_f64": ([_P, _P, _I32, _I32, _I32, _P, _P], None),
    "or_spmv_ell_f32": ([_P, _P, _I32, _I32, _P, _P], None),
    "or_spmv_ell_f64": ([_P, _P, _I32, _I32, _P, _P], None),
    "or_truth_csr_f32": ([_P, _P, _P, _P, _P, _P, _I32], None),
    "or_truth_csr_f64": ([_P, _P, _P, _P, _P, _P, _I32], None),
    "or_static_nnz": ([_P, _I32, _I32, _P, _P], None),
    "or_par_spmv_csr_f32": ([C.c_int, _P, _P, _P, _P, _P, _I32], None),
    "or_par_spmv_csr_f64": ([C.c_int, _P, _P, _P, _P, _P, _I32], None),
    "or_par_spmv_coo_f32": ([C.c_int, _P, _P, _P, _P, _P, _I32, _I64, _P], None),
    "or_par_spmv_coo_f64": ([C.c_int, _P, _P, _P, _P, _P, _I32, _I64, _P], None),
    "or_par_spmv_dia_f32": ([C.c_int, _P, _P, _I32, _I32, _I32, _P, _P], None),
    "or_par_spmv_dia_f64": ([C.c_int, _P, _P, _I32, _I32, _I32, _P, _P], None),
    "or_par_spmv_ell_f32": ([C.c_int, _P, _P, _I32, _I32, _P, _P], None),
    "or_par_spmv_ell_f64": ([C.c_int, _P, _P, _I32, _I32, _P, _P], None),
    "or_par_spmv_dia_rows_f32": ([C.c_int, _P, _P, _I32, _I32, _P, _P], None),
    "or_par_spmv_dia_rows_f64": ([C.c_int, _P, _P, _I32, _I32, _P, _P], None),
    "or_par_spmv_ell_rows_f32": ([C.c_int, _P, _P, _I32, _I32, _P, _P], None),
    "or_par_spmv_ell_rows_f64": ([C.c_int, _P, _P, _I32, _I32, _P, _P], None),
    "or_coo_csr": ([C.c_int, _P, _P, _P, _I32, _I64, _P, _P, _P], None),
    "or_coo_csc": ([C.c_int, _P, _P, _P, _I32, _I64, _P, _P, _P], None),
    "or_num_cols": ([_P, _I32], _I32),
    "or_format_admitted": ([_I64, _I64, _I64], C.c_int),
    "or_csr_ell": ([C.c_int, _P, _P, _P, _I32, _I32, _P, _P], None),
    "or_num_diags": ([_P, _P, _I32, _P], _I32),
    "or_csr_dia": ([C.c_int, _P, _P, _P, _I32, _I32, _I32, _P, _P], None),
    "or_quick_sort_coo": ([C.c_int, _P, _P, _P, _I64, _I64], None),
    "or_level_sets": ([C.c_int, _P, _P, _P, _I32, _P, _P, _P, _P, _P, _P, _P], _I32),
    "or_spts_csr_f32": ([_P, _P, _P, _P, _P, _I32], None),
    "or_spts_csr_f64": ([_P, _P, _P, _P, _P, _I32], None),
    "or_spts_syncfree_f32": ([_P, _P, _P, _P, _P, _I32], None),
    "or_spts_syncfree_f64": ([_P, _P, _P, _P, _P, _I32], None),
    "or_truth_spts": ([C.c_int, _P, _P, _P, _P, _P, _I32], None),
    "or_par_spts_level_f32": ([C.c_int, _P, _I32, _P, _P, _P, _P, _P, _I32], None),
    "or_par_spts_level_f64": ([C.c_int, _P, _I32, _P, _P, _P, _P, _P, _I32], None),
    "or_par_spts_syncfree_f32": ([C.c_int, _P, _P, _P, _P, _P, _I32, _P], C.c_int),
    "or_par_spts_syncfree_f64": ([C.c_int, _P, _P, _P, _P, _P, _I32, _P], C.c_int),
    "or_count_nonzeros": ([C.c_int, _P, _I64], _I64),
    "or_copy_nonzeros_coo": ([C.c_int, _P, _P, _P, _I64, _P, _P, _P], _I64),
    "or_copy_nonzeros_csr": ([C.c_int, _P, _P, _P, _I32, _P, _P, _P], None),
    "or_count_nonzeros_dia": ([C.c_int, _P, _P, _I32, _I32, _I32, _P, _P], None),
    "or_copy_nonzeros_dia": ([C.c_int, _P, _P, _I32, _I32, _I32, _P, _P], None),
    "or_count_nonzeros_ell": ([C.c_int, _P, _I32, _I32, _P, _P], None),
    "or_copy_nonzeros_ell": ([C.c_int, _P, _P, _I32, _I32, _P, _P], None),
    "or_transpose_csr": ([C.c_int, _P, _P, _P, _I32, _I64, _P, _P, _P], None),
    "or_transpose_dia": ([C.c_int, _P, _P, _I32, _I32, _I32, _P, _P], None),
    "or_count_transpose_cols_ell": ([C.c_int, _P, _P, _I32, _I32], _I32),
    "or_transpose_ell": ([C.c_int, _P, _P, _I32, _I32, _P, _P], None),
    "or_map": ([C.c_int, C.c_int, C.c_int, C.c_double, _P, _P, _I64], None),
    "or_map_dia": ([C.c_int, C.c_int, C.c_double, _P, _P, _P, _I32, _I32, _I32], None),
    "or_fletcher_f32": ([_P, _I64], _I64),
    "or_fletcher_f64": ([_P, _I64], _I64),
    "or_spts_csc": ([C.c_int, _P, _P, _P, _P, _P, _I32], None),
    "or_diagonal_coo": ([C.c_int, _I32, _P, _P, _P, _P, _I32, _I64], None),
    "or_min_coo": ([C.c_int, _I32, _P, _P, _P, _I32, _I64], None),
    "or_sum_coo_rows": ([C.c_int, _I32, _P, _P, _P, _I32, _I64], None),
    "or_sort_rows_by_nnz": ([C.c_int, _P, _P, _P, _I32, _P, _P, _P, _P, _P, _P], None),
    "or_unpermute_rows": ([C.c_int, _P, _P, _P, _I32], None),
    "or_csr_locality_index": ([_P, _P, _I32, _I64], C.c_double),
    "or_reorder_nn": ([C.c_int, _P, _P, _P, _I32, C.c_int, _P, _P, _P, _P, _P, _P], None),
    "or_reorder_nn_ex": ([C.c_int, C.c_int, _P, _P, _P, _I32, C.c_int, _P, _P, _P, _P, _P, _P],
                         None),
    "or_mm_read": ([_P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P], C.c_int),
    "or_mm_coo": ([C.c_int, C.c_int, _I32, _I32, _I64, _I64, _I64, _P, _P, _P, _P, _P, _P],
                  _I64),
}

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in _SIG.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data if a is not None else None


def _sfx(dtype) -> str:
    dt = np.dtype(dtype)
    if dt == np.float32:
        return "f32"
    if dt == np.float64:
        return "f64"
    raise TypeError(dt)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


# ------------------------------------------------------------------ SpMV

def spmv_csr(row_ptr, col, val, x, y):
    """y + A x in the reference's serial order; returns a new array."""
    y = np.array(y, dtype=val.dtype, copy=True)
    row_ptr, col, x = _i32(row_ptr), _i32(col), np.ascontiguousarray(x, val.dtype)
    getattr(lib(), "or_spmv_csr_" + _sfx(val.dtype))(
        _p(row_ptr), _p(col), _p(val), _p(x), _p(y), row_ptr.size - 1)
    return y


def spmv_coo(row, col, val, x, y):
    y = np.array(y, dtype=val.dtype, copy=True)
    row, col, x = _i32(row), _i32(col), np.ascontiguousarray(x, val.dtype)
    getattr(lib(), "or_spmv_coo_" + _sfx(val.dtype))(
        _p(row), _p(col), _p(val), _p(x), _p(y), row.size)
    return y


def spmv_dia(offset, data, N, x, y, stride=None):
    y = np.array(y, dtype=data.dtype, copy=True)
    offset, x = _i32(offset), np.ascontiguousarray(x, data.dtype)
    stride = N if stride is None else stride
    getattr(lib(), "or_spmv_dia_" + _sfx(data.dtype))(
        _p(offset), _p(data), N, offset.size, stride, _p(x), _p(y))
    return y


def spmv_ell(indices, data, N, nc, x, y):
    y = np.array(y, dtype=data.dtype, copy=True)
    indices, x = _i32(indices), np.ascontiguousarray(x, data.dtype)
    getattr(lib(), "or_spmv_ell_" + _sfx(data.dtype))(
        _p(indices), _p(data), N, nc, _p(x), _p(y))
    return y


def truth_csr(row_ptr, col, val, x, y0=None):
    """Extended-precision y0 + A x (float64 result)."""
    row_ptr, col = _i32(row_ptr), _i32(col)
    out = np.empty(row_ptr.size - 1, dtype=np.float64)
    x = np.ascontiguousarray(x, val.dtype)
    y0c = None if y0 is None else np.ascontiguousarray(y0, val.dtype)
    getattr(lib(), "or_truth_csr_" + _sfx(val.dtype))(
        _p(row_ptr), _p(col), _p(val), _p(x), _p(y0c), _p(out), row_ptr.size - 1)
    return out


def static_nnz(row_ptr, nw):
    row_ptr = _i32(row_ptr)
    rs = np.zeros(nw, np.int32)
    re = np.zeros(nw, np.int32)
    lib().or_static_nnz(_p(row_ptr), row_ptr.size - 1, nw, _p(rs), _p(re))
    return rs, re


def par_spmv_csr(nthreads, row_ptr, col, val, x, y):
    """Parallel CPU baseline; updates y in place."""
    getattr(lib(), "or_par_spmv_csr_" + _sfx(val.dtype))(
        nthreads, _p(row_ptr), _p(col), _p(val), _p(x), _p(y), row_ptr.size - 1)


def par_spmv_coo(nthreads, row, col, val, x, y, N, wy):
    getattr(lib(), "or_par_spmv_coo_" + _sfx(val.dtype))(
        nthreads, _p(row), _p(col), _p(val), _p(x), _p(y), N, row.size, _p(wy))


def par_spmv_dia(nthreads, offset, data, N, x, y):
    getattr(lib(), "or_par_spmv_dia_" + _sfx(data.dtype))(
        nthreads, _p(offset), _p(data), N, offset.size, N, _p(x), _p(y))


def par_spmv_ell(nthreads, indices, data, N, nc, x, y):
    getattr(lib(), "or_par_spmv_ell_" + _sfx(data.dtype))(
        nthreads, _p(indices), _p(data), N, nc, _p(x), _p(y))


def par_spmv_dia_rows(nthreads, offset, data_rows, N, x, y):
    """Parallel CPU baseline over row-by-row DIA data (data_rows[i*nd + d]);
    updates y in place."""
    getattr(lib(), "or_par_spmv_dia_rows_" + _sfx(data_rows.dtype))(
        nthreads, _p(offset), _p(data_rows), N, offset.size, _p(x), _p(y))


def par_spmv_ell_rows(nthreads, ind_rows, data_rows, N, nc, x, y):
    """Parallel CPU baseline over row-by-row ELL slots; updates y in place."""
    getattr(lib(), "or_par_spmv_ell_rows_" + _sfx(data_rows.dtype))(
        nthreads, _p(ind_rows), _p(data_rows), N, nc, _p(x), _p(y))


# ------------------------------------------------------------------ conversions

def coo_csr(row, col, val, N):
    row, col = _i32(row), _i32(col)
    val = np.ascontiguousarray(val)
    nnz = row.size
    rp = np.zeros(N + 1, np.int32)
    c = np.zeros(nnz, np.int32)
    v = np.zeros(nnz, val.dtype)
    lib().or_coo_csr(val.dtype.itemsize, _p(row), _p(col), _p(val), N, nnz, _p(rp), _p(c), _p(v))
    return rp, c, v


def coo_csc(row, col, val, ncols):
    row, col = _i32(row), _i32(col)
    val = np.ascontiguousarray(val)
    nnz = row.size
    cp = np.zeros(ncols + 1, np.int32)
    r = np.zeros(nnz, np.int32)
    v = np.zeros(nnz, val.dtype)
    lib().or_coo_csc(val.dtype.itemsize, _p(row), _p(col), _p(val), ncols, nnz, _p(cp), _p(r),
                     _p(v))
    return cp, r, v


def num_cols(row_ptr):
    row_ptr = _i32(row_ptr)
    return int(lib().or_num_cols(_p(row_ptr), row_ptr.size - 1))


def format_admitted(width, N, nnz) -> bool:
    return bool(lib().or_format_admitted(int(width), int(N), int(nnz)))


def csr_ell(row_ptr, col, val):
    """Returns (indices, data, nc) or None when the admission test refuses."""
    row_ptr, col = _i32(row_ptr), _i32(col)
    N = row_ptr.size - 1
    nc = num_cols(row_ptr)
    if not format_admitted(nc, N, col.size):
        return None
    ind = np.zeros(nc * N, np.int32)
    dat = np.zeros(nc * N, val.dtype)
    lib().or_csr_ell(val.dtype.itemsize, _p(row_ptr), _p(col), _p(val), N, nc, _p(ind), _p(dat))
    return ind, dat, nc


def num_diags(row_ptr, col):
    row_ptr, col = _i32(row_ptr), _i32(col)
    stride = np.zeros(1, np.int32)
    nd = lib().or_num_diags(_p(row_ptr), _p(col), row_ptr.size - 1, _p(stride))
    return int(nd), int(stride[0])


def csr_dia(row_ptr, col, val):
    """Returns (offset, data, nd, stride) or None when refused."""
    row_ptr, col = _i32(row_ptr), _i32(col)
    N = row_ptr.size - 1
    nd, stride = num_diags(row_ptr, col)
    if not format_admitted(nd, stride, col.size):
        return None
    off = np.zeros(nd, np.int32)
    dat = np.zeros(nd * stride, val.dtype)
    lib().or_csr_dia(val.dtype.itemsize, _p(row_ptr), _p(col), _p(val), N, nd, stride, _p(off),
                     _p(dat))
    return off, dat, nd, stride


def quick_sort_coo(row, col, val):
    row, col = _i32(row).copy(), _i32(col).copy()
    val = np.array(val, copy=True)
    if row.size:
        lib().or_quick_sort_coo(val.dtype.itemsize, _p(row), _p(col), _p(val), 0, row.size - 1)
    return row, col, val


# ------------------------------------------------------------------ SpTS

def level_sets(row_ptr, col, val):
    """Returns dict(level, level_ptr, permutation, order, row_ptr, col, val, nlevels)."""
    row_ptr, col = _i32(row_ptr), _i32(col)
    val = np.ascontiguousarray(val)
    N = row_ptr.size - 1
    level = np.zeros(N, np.int32)
    level_ptr = np.zeros(N + 2, np.int32)
    perm = np.zeros(N, np.int32)
    order = np.zeros(N, np.int32)
    nr = np.zeros(N + 1, np.int32)
    nc = np.zeros(col.size, np.int32)
    nv = np.zeros(col.size, val.dtype)
    nl = lib().or_level_sets(val.dtype.itemsize, _p(row_ptr), _p(col), _p(val), N, _p(level),
                             _p(level_ptr), _p(perm), _p(order), _p(nr), _p(nc), _p(nv))
    return dict(level=level, level_ptr=level_ptr[:nl + 1].copy(), permutation=perm, order=order,
                row_ptr=nr, col=nc, val=nv, nlevels=int(nl))


def _spts_args(row_ptr, col, val, b):
    """Contiguous operands, held by the caller for the duration of the call."""
    val = np.ascontiguousarray(val)
    return _i32(row_ptr), _i32(col), val, np.ascontiguousarray(b, val.dtype)


def spts_csr(row_ptr, col, val, b):
    rp, c, v, bb = _spts_args(row_ptr, col, val, b)
    y = np.zeros(rp.size - 1, v.dtype)
    getattr(lib(), "or_spts_csr_" + _sfx(v.dtype))(_p(rp), _p(c), _p(v), _p(bb), _p(y),
                                                    rp.size - 1)
    return y


def spts_syncfree(row_ptr, col, val, b):
    rp, c, v, bb = _spts_args(row_ptr, col, val, b)
    y = np.zeros(rp.size - 1, v.dtype)
    getattr(lib(), "or_spts_syncfree_" + _sfx(v.dtype))(_p(rp), _p(c), _p(v), _p(bb), _p(y),
                                                         rp.size - 1)
    return y


def truth_spts(row_ptr, col, val, b):
    rp, c, v, bb = _spts_args(row_ptr, col, val, b)
    y = np.zeros(rp.size - 1, np.float64)
    lib().or_truth_spts(v.dtype.itemsize, _p(rp), _p(c), _p(v), _p(bb), _p(y), rp.size - 1)
    return y


def par_spts_level(nthreads, level_ptr, row_ptr, col, val, b, y):
    getattr(lib(), "or_par_spts_level_" + _sfx(val.dtype))(
        nthreads, _p(level_ptr), level_ptr.size - 1, _p(row_ptr), _p(col), _p(val), _p(b), _p(y),
        row_ptr.size - 1)


def par_spts_syncfree(nthreads, row_ptr, col, val, b, y, flag=None):
    """Parallel sync-free CPU baseline into y (in place); flag is an int32[N]
    work array (allocated when None).  Raises if a bounded wait ran out."""
    if flag is None:
        flag = np.zeros(row_ptr.size - 1, np.int32)
    st = getattr(lib(), "or_par_spts_syncfree_" + _sfx(val.dtype))(
        nthreads, _p(row_ptr), _p(col), _p(val), _p(b), _p(y), row_ptr.size - 1, _p(flag))
    if st != 0:
        raise RuntimeError("or_par_spts_syncfree: a dependency wait ran out")


def fletcher(y):
    y = np.ascontiguousarray(y)
    return int(getattr(lib(), "or_fletcher_" + _sfx(y.dtype))(_p(y), y.size))


# ------------------------------------------------------------------ structure ops

def count_nonzeros(val):
    val = np.ascontiguousarray(val)
    return int(lib().or_count_nonzeros(val.dtype.itemsize, _p(val), val.size))


def copy_nonzeros_coo(row, col, val):
    row, col, val = _i32(row), _i32(col), np.ascontiguousarray(val)
    n = count_nonzeros(val)
    orow, ocol, oval = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(n, val.dtype)
    lib().or_copy_nonzeros_coo(val.dtype.itemsize, _p(row), _p(col), _p(val), row.size, _p(orow),
                               _p(ocol), _p(oval))
    return orow, ocol, oval


def copy_nonzeros_csr(row_ptr, col, val):
    row_ptr, col, val = _i32(row_ptr), _i32(col), np.ascontiguousarray(val)
    n = count_nonzeros(val)
    orp, ocol, oval = np.zeros(row_ptr.size, np.int32), np.zeros(n, np.int32), np.zeros(n, val.dtype)
    lib().or_copy_nonzeros_csr(val.dtype.itemsize, _p(row_ptr), _p(col), _p(val), row_ptr.size - 1,
                               _p(orp), _p(ocol), _p(oval))
    return orp, ocol, oval


def nonzeros_dia(offset, data, N, stride=None):
    offset, data = _i32(offset), np.ascontiguousarray(data)
    stride = N if stride is None else stride
    cd, cnt = np.zeros(1, np.int32), np.zeros(1, np.int64)
    lib().or_count_nonzeros_dia(data.dtype.itemsize, _p(offset), _p(data), offset.size, stride, N,
                                _p(cd), _p(cnt))
    ooff = np.zeros(int(cd[0]), np.int32)
    odat = np.zeros(int(cd[0]) * stride, data.dtype)
    lib().or_copy_nonzeros_dia(data.dtype.itemsize, _p(offset), _p(data), offset.size, stride, N,
                               _p(ooff), _p(odat))
    return int(cd[0]), int(cnt[0]), ooff, odat


def nonzeros_ell(data, indices, nc, N):
    data, indices = np.ascontiguousarray(data), _i32(indices)
    cc, cnt = np.zeros(1, np.int32), np.zeros(1, np.int64)
    lib().or_count_nonzeros_ell(data.dtype.itemsize, _p(data), nc, N, _p(cc), _p(cnt))
    onc = int(cc[0])
    od, oi = np.zeros(onc * N, data.dtype), np.zeros(onc * N, np.int32)
    lib().or_copy_nonzeros_ell(data.dtype.itemsize, _p(data), _p(indices), nc, N, _p(od), _p(oi))
    return onc, int(cnt[0]), od, oi


def transpose_csr(row_ptr, col, val):
    row_ptr, col, val = _i32(row_ptr), _i32(col), np.ascontiguousarray(val)
    N = row_ptr.size - 1
    orp, ocol, oval = np.zeros(N + 1, np.int32), np.zeros(col.size, np.int32), np.zeros(col.size, val.dtype)
    lib().or_transpose_csr(val.dtype.itemsize, _p(row_ptr), _p(col), _p(val), N, col.size, _p(orp),
                           _p(ocol), _p(oval))
    return orp, ocol, oval


def transpose_dia(offset, data, N, stride=None):
    offset, data = _i32(offset), np.ascontiguousarray(data)
    stride = N if stride is None else stride
    ooff, odat = np.zeros(offset.size, np.int32), np.zeros(data.size, data.dtype)
    lib().or_transpose_dia(data.dtype.itemsize, _p(offset), _p(data), offset.size, stride, N,
                           _p(ooff), _p(odat))
    return ooff, odat


def transpose_ell(data, indices, nc, N):
    data, indices = np.ascontiguousarray(data), _i32(indices)
    onc = int(lib().or_count_transpose_cols_ell(data.dtype.itemsize, _p(data), _p(indices), nc, N))
    od, oi = np.zeros(onc * N, data.dtype), np.zeros(onc * N, np.int32)
    lib().or_transpose_ell(data.dtype.itemsize, _p(data), _p(indices), nc, N, _p(od), _p(oi))
    return onc, od, oi


def map_values(values, kind, op, p=0.0):
    """kind 0: COO/CSR kernels, 1: DIA/ELL kernels."""
    a = np.ascontiguousarray(values)
    out = np.empty_like(a)
    lib().or_map(a.dtype.itemsize, kind, op, float(p), _p(a), _p(out), a.size)
    return out


def map_dia(offset, data, N, op, p=0.0, out=None, stride=None):
    offset, data = _i32(offset), np.ascontiguousarray(data)
    stride = N if stride is None else stride
    out = np.zeros_like(data) if out is None else np.array(out, copy=True)
    lib().or_map_dia(data.dtype.itemsize, op, float(p), _p(offset), _p(data), _p(out), offset.size,
                     stride, N)
    return out


# ------------------------------------------------------------------ Matrix Market

def mm_read(text: bytes) -> dict:
    """read_matrix_MM_files on the file's bytes: header, 1-based entries, nnz."""
    buf = np.frombuffer(bytes(text), dtype=np.uint8)
    nr, nc, ne = C.c_int64(), C.c_int64(), C.c_int64()
    field, sym = C.c_int32(), C.c_int32()
    nnz = C.c_int64()
    L = lib()
    if L.or_mm_read(_p(buf), buf.size, C.byref(nr), C.byref(nc), C.byref(ne), C.byref(field),
                    C.byref(sym), None, None, None, None):
        raise ValueError("entries : invalid length, cannot allocate")
    row = np.zeros(ne.value, np.int32)
    col = np.zeros(ne.value, np.int32)
    val = np.zeros(ne.value, np.float64)
    if L.or_mm_read(_p(buf), buf.size, C.byref(nr), C.byref(nc), C.byref(ne), C.byref(field),
                    C.byref(sym), _p(row), _p(col), _p(val), C.byref(nnz)):
        raise ValueError("nnz : invalid length, cannot allocate")
    return dict(nrows=nr.value, ncols=nc.value, nentries=ne.value, field=field.value,
                symmetric=sym.value, row=row, col=col, val=val, nnz=nnz.value)


def mm_coo(info: dict, dtype=np.float32, lower=False):
    """create_COO_from_MM (lower=False) or create_LCOO_from_MM (lower=True),
    sorted by quick_sort_COO.  Returns (row, col, val)."""
    dt = np.dtype(dtype)
    cap = info["nnz"] if not lower else info["nrows"] + 2 * info["nentries"]
    row = np.zeros(max(cap, 1), np.int32)
    col = np.zeros(max(cap, 1), np.int32)
    val = np.zeros(max(cap, 1), dt)
    n = lib().or_mm_coo(dt.itemsize, int(lower), info["field"], info["symmetric"], info["nrows"],
                        info["nentries"], info["nnz"], _p(info["row"]), _p(info["col"]),
                        _p(info["val"]), _p(row), _p(col), _p(val))
    return row[:n], col[:n], val[:n]


# ------------------------------------------------------------------ COO reductions

def diagonal_coo(k, row, col, val, N):
    row, col, val = _i32(row), _i32(col), np.ascontiguousarray(val)
    out = np.zeros(max(N - abs(k), 0), val.dtype)
    lib().or_diagonal_coo(val.dtype.itemsize, k, _p(row), _p(col), _p(val), _p(out), N, row.size)
    return out


def min_coo(axis, row, val, N):
    row, val = _i32(row), np.ascontiguousarray(val)
    out = np.zeros(N, val.dtype)
    lib().or_min_coo(val.dtype.itemsize, axis, _p(row), _p(val), _p(out), N, row.size)
    return out


def sum_coo_rows(axis, row, val, N):
    row, val = _i32(row), np.ascontiguousarray(val)
    out = np.zeros(N, val.dtype)
    lib().or_sum_coo_rows(val.dtype.itemsize, axis, _p(row), _p(val), _p(out), N, row.size)
    return out


# ------------------------------------------------------------------ row reordering

def sort_rows_by_nnz(row_ptr, col, val):
    row_ptr, col, val = _i32(row_ptr), _i32(col), np.ascontiguousarray(val)
    N = row_ptr.size - 1
    nrp = np.zeros(N + 1, np.int32)
    ncol = np.zeros(col.size, np.int32)
    nval = np.zeros(col.size, val.dtype)
    npr = np.zeros(N, np.int32)
    perm = np.zeros(N, np.int32)
    small = np.zeros(4, np.int32)
    lib().or_sort_rows_by_nnz(val.dtype.itemsize, _p(row_ptr), _p(col), _p(val), N, _p(nrp),
                              _p(ncol), _p(nval), _p(npr), _p(perm), _p(small))
    return dict(row_ptr=nrp, col=ncol, val=nval, nnz_per_row=npr, permutation=perm,
                small_rows=small)


def unpermute_rows(permutation, y):
    permutation, y = _i32(permutation), np.ascontiguousarray(y)
    out = np.zeros_like(y)
    lib().or_unpermute_rows(y.dtype.itemsize, _p(permutation), _p(y), _p(out), y.size)
    return out


def reorder_nn(row_ptr, col, val, w=16, perm_in=None, list_bytes=4):
    """dict(walk, permutation, row_ptr, col, val) of reorder_NN.  list_bytes:
    4 = the FP32 build's float32 similarity list (the device's rule), 8 = the
    FP64 build's double list."""
    row_ptr, col, val = _i32(row_ptr), _i32(col), np.ascontiguousarray(val)
    N = row_ptr.size - 1
    pin = None if perm_in is None else _i32(perm_in)
    walk, perm = np.zeros(N, np.int32), np.zeros(N, np.int32)
    nrp = np.zeros(N + 1, np.int32)
    ncol, nval = np.zeros(col.size, np.int32), np.zeros(col.size, val.dtype)
    lib().or_reorder_nn_ex(val.dtype.itemsize, int(list_bytes), _p(row_ptr), _p(col), _p(val), N,
                           int(w), _p(pin), _p(walk), _p(perm), _p(nrp), _p(ncol), _p(nval))
    return dict(walk=walk, permutation=perm, row_ptr=nrp, col=ncol, val=nval)


def csr_locality_index(row_ptr, col):
    row_ptr, col = _i32(row_ptr), _i32(col)
    return lib().or_csr_locality_index(_p(row_ptr), _p(col), row_ptr.size - 1, col.size)


def spts_csc(col_ptr, row, val, x):
    col_ptr, row, val = _i32(col_ptr), _i32(row), np.ascontiguousarray(val)
    x = np.ascontiguousarray(x, val.dtype)
    y = np.zeros(col_ptr.size - 1, val.dtype)
    lib().or_spts_csc(val.dtype.itemsize, _p(col_ptr), _p(row), _p(val), _p(x), _p(y),
                      col_ptr.size - 1)
    return y
