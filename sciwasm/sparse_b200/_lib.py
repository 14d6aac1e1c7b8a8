"""ctypes binding of libsparse_b200.so (the C ABI declared in include/sparse_b200.h).

The library is loaded from this package directory.  There is no fallback: if
the shared object is missing, or a call returns an error status, the call
raises.  Every array argument is a device pointer passed as an integer.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsparse_b200.so")

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
SZ = C.c_size_t

SB_OK = 0
SB_EINVAL = -1
SB_ENOMEM = -2
SB_EREFUSED = -3
SB_ETIMEOUT = -4
SB_ECUDA = -5
SB_ENODEV = -6
SB_EALIGN = -7
SB_COO_ROWS_SORTED = 1

SB_F32 = 0
SB_F64 = 1
SB_BF16 = 2

SB_SPTS_LEVEL = 0
SB_SPTS_SYNCFREE = 1
SB_SPTS_HYBRID = 2
SB_SPTS_ACC_NATIVE = 0
SB_SPTS_ACC_F64 = 1

# name -> argtypes (all functions return int status unless listed in _RESTYPE)
SIGNATURES: dict[str, list] = {
    "sb_version": [],
    "sb_last_error": [],
    "sb_status_string": [C.c_int],
    "sb_device_count": [C.POINTER(C.c_int)],
    "sb_set_device": [C.c_int],
    "sb_malloc": [C.POINTER(P), SZ],
    "sb_free": [P],
    "sb_host_alloc": [C.POINTER(P), SZ],
    "sb_host_free": [P],
    "sb_memcpy_htod": [P, P, SZ, P],
    "sb_memcpy_dtoh": [P, P, SZ, P],
    "sb_memcpy_dtod": [P, P, SZ, P],
    "sb_memset": [P, C.c_int, SZ, P],
    "sb_stream_create": [C.POINTER(P)],
    "sb_stream_create_priority": [C.POINTER(P), C.c_int],
    "sb_stream_priority_range": [C.POINTER(C.c_int), C.POINTER(C.c_int)],
    "sb_stream_destroy": [P],
    "sb_stream_synchronize": [P],
    "sb_mem_info": [C.POINTER(SZ), C.POINTER(SZ)],
    "sb_device_status": [C.POINTER(C.c_int)],
    "sb_event_create": [C.POINTER(P)],
    "sb_event_destroy": [P],
    "sb_event_record": [P, P],
    "sb_event_query": [P],
    "sb_event_synchronize": [P],
    "sb_event_elapsed_ms": [P, P, C.POINTER(C.c_float)],
    "sb_stream_wait_event": [P, P],
    "sb_spmv_coo": [C.c_int, P, P, P, P, P, I32, I64, I32, P],
    "sb_spmv_coo_ex": [C.c_int, P, P, P, P, P, I32, I64, I32, I32, P],
    "sb_spmv_csr": [C.c_int, P, P, P, P, P, I32, I64, I32, P],
    "sb_spmv_dia": [C.c_int, P, P, I32, I32, I32, P, P, I32, P],
    "sb_spmv_ell": [C.c_int, P, P, I32, I32, P, P, I32, P],
    "sb_coo_csr": [C.c_int, P, P, P, I32, I64, P, P, P, P],
    "sb_num_cols": [P, I32, C.POINTER(I32), P],
    "sb_ell_admitted": [I64, I32, I64],
    "sb_csr_ell": [C.c_int, P, P, P, I32, I64, I32, P, P, P],
    "sb_num_diags": [P, P, I32, C.POINTER(I32), C.POINTER(I32), P],
    "sb_dia_admitted": [I64, I32, I64],
    "sb_csr_dia": [C.c_int, P, P, P, I32, I64, I32, I32, P, P, P],
    "sb_spts_analyze": [C.c_int, P, P, P, I32, I64, P, C.POINTER(P)],
    "sb_spts_plan_destroy": [P],
    "sb_spts_plan_info": [P, C.POINTER(I32), C.POINTER(I32)],
    "sb_spts_plan_analysis_ms": [P, C.POINTER(C.c_float)],
    "sb_spts_plan_levels": [P, P, P, P, P, P],
    "sb_spts_plan_reordered": [P, P, P, P, P],
    "sb_spts_solve": [P, C.c_int, C.c_int, P, P, P],
    "sb_spts_syncfree_csr": [C.c_int, P, P, P, I32, P, P, I64, P],
    "sb_spts_syncfree_csr_noalloc": [C.c_int, P, P, P, I32, P, P, I64, P],
    "sb_count_nonzeros": [C.c_int, P, I64, C.POINTER(I64), P],
    "sb_copy_nonzeros_coo": [C.c_int, P, P, P, I64, P, P, P, P],
    "sb_copy_nonzeros_csr": [C.c_int, P, P, P, I32, I64, P, P, P, P],
    "sb_count_nonzeros_dia": [C.c_int, P, P, I32, I32, I32, C.POINTER(I32), C.POINTER(I64), P],
    "sb_copy_nonzeros_dia": [C.c_int, P, P, I32, I32, I32, P, P, P],
    "sb_count_nonzeros_ell": [C.c_int, P, I32, I32, C.POINTER(I32), C.POINTER(I64), P],
    "sb_copy_nonzeros_ell": [C.c_int, P, P, I32, I32, I32, P, P, P],
    "sb_transpose_coo": [C.c_int, P, P, P, I64, P, P, P, P],
    "sb_transpose_csr": [C.c_int, P, P, P, I32, I64, P, P, P, P],
    "sb_transpose_dia": [C.c_int, P, P, I32, I32, I32, P, P, P],
    "sb_count_transpose_cols_ell": [C.c_int, P, P, I32, I32, C.POINTER(I32), P],
    "sb_transpose_ell": [C.c_int, P, P, I32, I32, I32, P, P, P],
    "sb_map_coo": [C.c_int, C.c_int, C.c_double, P, P, I64, P],
    "sb_map_ell": [C.c_int, C.c_int, C.c_double, P, P, I32, I32, P],
    "sb_map_dia": [C.c_int, C.c_int, C.c_double, P, P, P, I32, I32, I32, P],
}
class CsrOpts(C.Structure):
    _fields_ = [("kernel", I32), ("lanes_per_row", I32), ("unroll", I32), ("grid", I32)]


class BatchItem(C.Structure):
    _fields_ = [("row_ptr", P), ("col", P), ("val", P), ("x", P), ("y", P), ("N", I32),
                ("nrhs", I32), ("lanes", I32), ("flags", I32), ("nnz", I64), ("format", I32),
                ("width", I32)]


SB_FMT_CSR, SB_FMT_DIA, SB_FMT_ELL, SB_FMT_COO = 0, 1, 2, 3
SB_TUNE_MODEL, SB_TUNE_TIMED = 0, 1


class SpmvChoice(C.Structure):
    _fields_ = [("format", I32), ("csr", CsrOpts), ("ndiags", I32), ("ncols", I32),
                ("dia_admitted", I32), ("ell_admitted", I32), ("ms", C.c_float * 4),
                ("bytes", I64 * 4)]


class MMHeader(C.Structure):
    _fields_ = [("nrows", I64), ("ncols", I64), ("nentries", I64), ("field", I32),
                ("symmetric", I32), ("data_offset", I64)]


SB_MM_REAL, SB_MM_INTEGER, SB_MM_PATTERN, SB_MM_COMPLEX = 0, 1, 2, 3


class SptsBatchItem(C.Structure):
    _fields_ = [("plan", P), ("b", P), ("y", P), ("work", P)]


SIGNATURES.update({
    "sb_diagonal_coo": [C.c_int, I32, P, P, P, P, I32, I64, P],
    "sb_min_coo": [C.c_int, I32, P, P, P, P, I32, I64, P],
    "sb_sum_coo": [C.c_int, I32, P, P, P, P, I32, I64, P],
    "sb_sort_rows_by_nnz": [C.c_int, P, P, P, I32, I64, P, P, P, P, P, C.POINTER(I32), P],
    "sb_unpermute_rows": [C.c_int, P, P, P, I32, P],
    "sb_csr_locality_index": [P, P, I32, I64, C.POINTER(C.c_double), P],
    "sb_reorder_nn": [C.c_int, P, P, P, I32, I64, I32, P, P, P, P, P, P, P],
    "sb_coo_csc": [C.c_int, P, P, P, I32, I64, P, P, P, P],
    "sb_spts_csc": [C.c_int, P, P, P, I32, I64, P, P, P],
    "sb_mm_read_header": [P, SZ, C.POINTER(MMHeader)],
    "sb_mm_read_entries": [P, SZ, C.POINTER(MMHeader), P, P, P, I32],
    "sb_mm_coo": [C.c_int, C.c_int, C.POINTER(MMHeader), P, P, P, P, P, P, C.POINTER(I64), P],
    "sb_spts_plan_growth": [P, C.POINTER(C.c_double), P],
    "sb_spts_batch_create": [C.c_int, C.c_int, I32, C.POINTER(P)],
    "sb_spts_batch_destroy": [P],
    "sb_spts_batch_run": [P, C.POINTER(SptsBatchItem), I32, P],
    "sb_spts_batch_set_grid": [P, I32],
    "sb_batch_exec_create": [C.c_int, I32, C.POINTER(P)],
    "sb_batch_exec_destroy": [P],
    "sb_batch_exec_run": [P, C.POINTER(BatchItem), I32, P],
    "sb_convert_values": [C.c_int, P, C.c_int, P, I64, P],
    "sb_spmv_csr_ex": [C.c_int, P, P, P, P, P, I32, I64, I32, C.POINTER(CsrOpts), P],
    "sb_spmv_csr_allgather": [C.c_int, P, P, P, P, P, I32, I64, I64, P, I32,
                              C.POINTER(CsrOpts), P],
    "sb_gather_dot": [C.c_int, P, P, P, I64, P, P],
    "sb_gather_dot_rows": [C.c_int, P, P, P, I64, I32, I64, P, P],
    "sb_spmv_autotune": [C.c_int, P, P, P, P, I32, I64, I32, I32, C.POINTER(SpmvChoice), P],
    "sb_csr_coo": [C.c_int, P, P, P, I32, I64, P, P, P, P],
    "sb_csr_autotune": [C.c_int, P, P, P, P, I32, I64, I32, C.POINTER(CsrOpts),
                        C.POINTER(C.c_float), P],
})

_RESTYPE = {"sb_last_error": C.c_char_p, "sb_status_string": C.c_char_p}


class SparseError(RuntimeError):
    """A libsparse_b200 call returned a negative status."""

    def __init__(self, fn: str, status: int, message: str):
        super().__init__(f"{fn} failed with status {status}: {message}")
        self.fn = fn
        self.status = status


class RefusedError(SparseError):
    """The format admission test of csr_ell / csr_dia refused the matrix."""


_lib = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Load the shared object (once) and attach signatures."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m sciwasm.sparse_b200.build` "
                "(the CUDA path has no CPU fallback)")
        lib = C.CDLL(LIB_PATH)
        for name, argtypes in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = _RESTYPE.get(name, C.c_int)
        _lib = lib
        return lib


def declared_symbols() -> list[str]:
    return list(SIGNATURES)


def call(name: str, *args) -> int:
    """Call `name`; raise SparseError on a negative status, return the status."""
    lib = load()
    st = getattr(lib, name)(*args)
    if st < 0:
        msg = (lib.sb_last_error() or b"").decode(errors="replace")
        if st == SB_EREFUSED:
            raise RefusedError(name, st, msg)
        raise SparseError(name, st, msg)
    return st


def last_error() -> str:
    return (load().sb_last_error() or b"").decode(errors="replace")
