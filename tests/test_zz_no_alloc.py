"""The no-allocation sync-free solve, sb_spts_syncfree_csr_noalloc.

Some callers cannot allocate device memory when they solve: a serving process
that reserved its whole HBM budget for resident matrices up front, or an
embedding runtime that owns every device allocation.  This entry point keeps
its scratch (ready flags, row ticket, status word) in a fixed device array
inside the library instead.  The test calls it through the C ABI and checks
its output against the allocating entry point, sb_spts_syncfree_csr, on two
calls in a row (the shared array must be cleared between calls).  The file
name makes pytest collect it last; it passes alone and after the others.
"""
import ctypes

import numpy as np
import pytest

from conftest import TOL
from sciwasm.sparse_b200 import _lib, synth

pytestmark = pytest.mark.gpu

MAX_ROWS = 1 << 22


def _dev(arr):
    from sciwasm.sparse_b200.sparse import DeviceArray
    return DeviceArray.from_host(arr)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_noalloc_matches_allocating_entry_point_twice(gpu, dt):
    lib = _lib.load()
    code = _lib.SB_F32 if dt == np.float32 else _lib.SB_F64
    rp, col, val = synth.random_lower(200_000, seed=11, band=3000, dtype=dt)
    N = rp.size - 1
    d_rp, d_col, d_val = _dev(rp), _dev(col), _dev(val)
    for call in range(2):
        b = synth.uniform_vec(N, 20 + call, dtype=dt)
        d_b = _dev(b)
        ref_y = _dev(np.zeros(N, dt))
        new_y = _dev(np.full(N, np.nan, dt))
        st = lib.sb_spts_syncfree_csr(code, d_rp.ptr, d_col.ptr, d_val.ptr, N, d_b.ptr, ref_y.ptr,
                                      0, None)
        assert st == 0, lib.sb_last_error()
        st = lib.sb_spts_syncfree_csr_noalloc(code, d_rp.ptr, d_col.ptr, d_val.ptr, N, d_b.ptr,
                                              new_y.ptr, 0, None)
        assert st == 0, lib.sb_last_error()
        want, got = ref_y.to_host(), new_y.to_host()
        err = np.max(np.abs(got.astype(np.float64) - want)) / np.max(np.abs(want))
        assert err <= TOL[np.dtype(dt)], (call, err)
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), call


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_noalloc_matches_oracle_sync_free_order(gpu, oracle, dt):
    """Bit-identical to the oracle's restatement of the reference's sync-free
    kernel (subtract as you go, divide by the diagonal last)."""
    lib = _lib.load()
    code = _lib.SB_F32 if dt == np.float32 else _lib.SB_F64
    rp, col, val = synth.laplacian_3d_lower(40, dtype=dt)
    N = rp.size - 1
    d_rp, d_col, d_val = _dev(rp), _dev(col), _dev(val)
    for call in range(2):
        b = synth.uniform_vec(N, 30 + call, dtype=dt)
        y = _dev(np.full(N, np.nan, dt))
        d_b = _dev(b)  # held: a temporary's device buffer is freed as soon as it is dropped
        st = lib.sb_spts_syncfree_csr_noalloc(code, d_rp.ptr, d_col.ptr, d_val.ptr, N,
                                              d_b.ptr, y.ptr, 0, None)
        assert st == 0, lib.sb_last_error()
        want = oracle.spts_syncfree(rp, col, val, b)
        assert np.array_equal(y.to_host().view(np.uint8), want.view(np.uint8)), call


def test_noalloc_timeout_then_next_call_is_clean(gpu, oracle):
    """Row 2 lists itself before its diagonal, so its own ready flag is awaited
    and the bounded wait runs out: SB_ETIMEOUT.  The status word lives in the
    shared array, so the next call must clear it, and a good solve right after
    must match the oracle bit for bit."""
    lib = _lib.load()
    rp = np.array([0, 1, 3, 6], np.int32)
    col = np.array([0, 0, 1, 0, 2, 2], np.int32)
    val = np.array([2.0, 1.0, 4.0, 1.0, 1.0, 8.0])
    d = [_dev(a) for a in (rp, col, val, np.ones(3), np.zeros(3))]
    st = lib.sb_spts_syncfree_csr_noalloc(_lib.SB_F64, d[0].ptr, d[1].ptr, d[2].ptr, 3, d[3].ptr,
                                          d[4].ptr, 1 << 20, None)
    assert st == _lib.SB_ETIMEOUT, lib.sb_last_error()
    grp, gcol, gval = synth.laplacian_3d_lower(8)
    b = synth.uniform_vec(512, 2)
    y = _dev(np.zeros(512))
    g = [_dev(a) for a in (grp, gcol, gval, b)]  # held for the duration of the call
    st = lib.sb_spts_syncfree_csr_noalloc(_lib.SB_F64, g[0].ptr, g[1].ptr, g[2].ptr, 512,
                                          g[3].ptr, y.ptr, 0, None)
    assert st == 0, lib.sb_last_error()
    want = oracle.spts_syncfree(grp, gcol, gval, b)
    assert np.array_equal(y.to_host().view(np.uint8), want.view(np.uint8))


def test_noalloc_rejects_sizes_beyond_its_limit(gpu):
    lib = _lib.load()
    tiny = _dev(np.zeros(4, np.int32))
    st = lib.sb_spts_syncfree_csr_noalloc(_lib.SB_F64, tiny.ptr, tiny.ptr, tiny.ptr, MAX_ROWS + 1,
                                          tiny.ptr, tiny.ptr, 0, None)
    assert st == _lib.SB_EINVAL
    assert b"4194304" in lib.sb_last_error()
