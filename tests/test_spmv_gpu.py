"""SpMV parity on the GPU through the C ABI: CSR and COO within the stated
tolerance of the extended-precision truth (and of the oracle's serial order);
DIA and ELL bit-identical to the oracle (they keep the reference's per-row
order with separately rounded mul and add)."""
import numpy as np
import pytest

from conftest import TOL, rel_err
from sciwasm.sparse_b200 import synth

pytestmark = pytest.mark.gpu

DTYPES = [np.float32, np.float64]


def _mats(dt):
    out = {}
    out["laplacian256"] = synth.laplacian_2d(256, dtype=dt)
    out["banded"] = synth.banded(100_003, seed=1, dtype=dt)
    out["powerlaw"] = synth.power_law(40_000, seed=2, dtype=dt, cap=2000, sort_cols=False)
    # long rows spanning many warp tiles, rows of every short length, empty rows
    rng = np.random.default_rng(11)
    lens = np.concatenate([[5000, 0, 0, 1, 2, 3, 4, 700], rng.integers(0, 9, 6000), [0, 0, 1]])
    N = lens.size
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = np.concatenate([np.sort(rng.choice(N, l, replace=False)) for l in lens]).astype(np.int32)
    out["ragged"] = (rp, col, rng.uniform(-1, 1, col.size).astype(dt))
    out["single"] = (np.array([0, 1], np.int32), np.array([0], np.int32), np.array([3.0], dt))
    out["many_empty"] = (np.concatenate([[0] * 5000, [1] * 5000, [3]]).astype(np.int32),
                         np.array([7, 1, 9999], np.int32), np.array([1.0, -2.0, 0.5], dt))
    return out


def _x_y(N, dt, seed=0):
    return (synth.uniform_vec(N, seed, dtype=dt), synth.uniform_vec(N, seed + 100, dtype=dt))


@pytest.mark.parametrize("dt", DTYPES)
def test_csr_parity(gpu, oracle, dt):
    for name, (rp, col, val) in _mats(dt).items():
        N = rp.size - 1
        x, y0 = _x_y(N, dt)
        A = gpu.csr_from_host(rp, col, val)
        xv, yv = gpu.vec_from_host(x), gpu.vec_from_host(y0)
        gpu.spmv(A, xv, yv)
        y = yv.array()
        truth = oracle.truth_csr(rp, col, val, x, y0)
        assert rel_err(y, truth) <= TOL[np.dtype(dt)], name
        ys = oracle.spmv_csr(rp, col, val, x, y0)
        assert rel_err(y, ys) <= 2 * TOL[np.dtype(dt)], name
        # rows without entries keep their exact bits
        empty = np.diff(rp) == 0
        assert np.array_equal(y[empty].view(np.uint8), y0[empty].view(np.uint8)), name


@pytest.mark.parametrize("dt", DTYPES)
def test_csr_inner_max_accumulates(gpu, oracle, dt):
    rp, col, val = synth.laplacian_2d(64, dtype=dt)
    N = rp.size - 1
    x, _ = _x_y(N, dt)
    A = gpu.csr_from_host(rp, col, val)
    xv, yv = gpu.vec_from_host(x), gpu.create_vec(N, 0, dt)
    gpu.spmv(A, xv, yv, inner_max=3)
    truth = 3.0 * oracle.truth_csr(rp, col, val, x)
    assert rel_err(yv.array(), truth) <= 3 * TOL[np.dtype(dt)]


@pytest.mark.parametrize("dt", DTYPES)
def test_csr_unaligned_pointers(gpu, oracle, dt):
    """Sub-array views whose col/val start off a 16-byte boundary take the
    scalar-load path and must give the same result."""
    from sciwasm.sparse_b200.sparse import DeviceArray, sparse_CSR_t
    rp, col, val = synth.power_law(5000, seed=4, dtype=dt, cap=300)
    N = rp.size - 1
    x, y0 = _x_y(N, dt, 3)
    colp = np.concatenate([[0], col]).astype(np.int32)
    valp = np.concatenate([[0], val]).astype(dt)
    dcol, dval = DeviceArray.from_host(colp), DeviceArray.from_host(valp)
    A = sparse_CSR_t(DeviceArray.from_host(rp), DeviceArray(col.size, np.int32, dcol.ptr + 4),
                     DeviceArray(val.size, dt, dval.ptr + np.dtype(dt).itemsize), N, col.size)
    xv, yv = gpu.vec_from_host(x), gpu.vec_from_host(y0)
    gpu.spmv(A, xv, yv)
    assert rel_err(yv.array(), oracle.truth_csr(rp, col, val, x, y0)) <= TOL[np.dtype(dt)]


@pytest.mark.parametrize("dt", DTYPES)
def test_coo_parity_sorted_and_unsorted(gpu, oracle, dt):
    for name, (rp, col, val) in _mats(dt).items():
        N = rp.size - 1
        row = synth.csr_to_coo_rows(rp)
        x, y0 = _x_y(N, dt, 5)
        truth = oracle.truth_csr(rp, col, val, x, y0)
        perm = np.random.default_rng(1).permutation(row.size)
        for r, c, v in ((row, col, val), (row[perm], col[perm], val[perm])):
            A = gpu.coo_from_host(r, c, v, N)
            # sorted rows take the kernel that adds whole rows without atomics
            assert A.rows_sorted == bool(np.all(np.diff(r) >= 0)), name
            xv, yv = gpu.vec_from_host(x), gpu.vec_from_host(y0)
            gpu.spmv(A, xv, yv)
            assert rel_err(yv.array(), truth) <= TOL[np.dtype(dt)], name


@pytest.mark.parametrize("dt", DTYPES)
def test_coo_rows_sorted_carried(gpu, oracle, dt):
    """Order-preserving operations keep a COO's rows_sorted flag (and its
    sorted-rows SpMV), transpose drops it; results stay within tolerance."""
    rp, col, val = synth.banded(50_021, half=4, seed=7, dtype=dt)
    val = val.copy()
    val[::7] = 0.0  # explicit zeros for eliminate_zeros to drop
    N = rp.size - 1
    row = synth.csr_to_coo_rows(rp)
    A = gpu.coo_from_host(row, col, val, N)
    assert A.rows_sorted
    x, y0 = _x_y(N, dt, 8)
    keep = val != 0
    B = gpu.eliminate_zeros(A)
    assert B.rows_sorted and B.nnz == int(keep.sum())
    Nb = np.concatenate([[0], np.cumsum(np.bincount(row[keep], minlength=N))]).astype(np.int32)
    cases = [(B, Nb, col[keep], val[keep]),
             (gpu.neg(A), rp, col, -val)]
    T = gpu.transpose(A)
    assert not T.rows_sorted
    for M, mrp, mcol, mval in cases:
        assert M.rows_sorted
        xv, yv = gpu.vec_from_host(x), gpu.vec_from_host(y0)
        gpu.spmv(M, xv, yv)
        assert rel_err(yv.array(), oracle.truth_csr(mrp, mcol, mval, x, y0)) <= TOL[np.dtype(dt)]


@pytest.mark.parametrize("dt", DTYPES)
def test_dia_ell_bitexact(gpu, oracle, dt):
    mats = _mats(dt)
    # 21 diagonals: above the counts with a compile-time specialised kernel
    mats["banded21"] = synth.banded(30_011, half=10, seed=4, dtype=dt)
    for name in ("laplacian256", "banded", "banded21"):
        rp, col, val = mats[name]
        N = rp.size - 1
        x, y0 = _x_y(N, dt, 9)
        off, dat, nd, stride = oracle.csr_dia(rp, col, val)
        A = gpu.dia_from_host(off, dat, N)
        xv, yv = gpu.vec_from_host(x), gpu.vec_from_host(y0)
        gpu.spmv(A, xv, yv, inner_max=2)
        want = oracle.spmv_dia(off, dat, N, x, oracle.spmv_dia(off, dat, N, x, y0))
        assert np.array_equal(yv.array().view(np.uint8), want.view(np.uint8)), name
        ind, edat, nc = oracle.csr_ell(rp, col, val)
        E = gpu.ell_from_host(ind, edat, nc, N)
        yv2 = gpu.vec_from_host(y0)
        gpu.spmv(E, xv, yv2)
        want = oracle.spmv_ell(ind, edat, N, nc, x, y0)
        assert np.array_equal(yv2.array().view(np.uint8), want.view(np.uint8)), name


def test_empty_row_semantics(gpu, oracle):
    import json
    import os
    k = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                    "kat_reference_semantics.json")))[
        "csr_empty_row_keeps_negative_zero"]
    y0 = np.array(k["y0_bits_f32"], np.uint32).view(np.float32)
    x = np.array(k["x"], np.float32)
    A = gpu.csr_from_host(k["row_ptr"], k["col"], np.array(k["val"], np.float32))
    xv, yv = gpu.vec_from_host(x), gpu.vec_from_host(y0)
    gpu.spmv(A, xv, yv)
    assert yv.array().view(np.uint32).tolist() == \
        np.array(k["csr_y"], np.float32).view(np.uint32).tolist()
    E = gpu.ell_from_host(k["ell_indices"], np.array(k["ell_data"], np.float32), 1, 2)
    yv = gpu.vec_from_host(y0)
    gpu.spmv(E, xv, yv)
    assert yv.array().view(np.uint32).tolist() == \
        np.array(k["ell_y"], np.float32).view(np.uint32).tolist()


def test_zero_sized_calls_are_noops(gpu):
    A = gpu.csr_from_host(np.zeros(4, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32))
    xv, yv = gpu.create_vec(3, 1.0), gpu.create_vec(3, 2.0)
    gpu.spmv(A, xv, yv)
    assert yv.array().tolist() == [2.0, 2.0, 2.0]


@pytest.mark.parametrize("storage", ["f32", "f64", "bf16"])
@pytest.mark.parametrize("tiles", [1, 4, 16])
def test_csr_nonzero_tile_kernel(gpu, oracle, storage, tiles):
    """Kernel 2 (row-aligned nonzero ranges, 256-nonzero tiles): within the
    tolerance of the exact result, rows without entries keep their bits, and
    two runs give identical bits (every row is written once, no atomics)."""
    from sciwasm.sparse_b200 import _lib
    dt = np.float64 if storage == "f64" else np.float32
    for name, (rp, col, val) in _mats(dt).items():
        N = rp.size - 1
        x, y0 = _x_y(N, dt)
        A = gpu.csr_from_host(rp, col, val)
        vals = val
        if storage == "bf16":
            A = gpu.csr_with_storage(A, "bf16")
            vals = (A.val_array().astype(np.uint32) << 16).view(np.float32)
        A.opts = _lib.CsrOpts(2, 0, tiles, 0)
        outs = []
        for _ in range(2):
            xv, yv = gpu.vec_from_host(x), gpu.vec_from_host(y0)
            gpu.spmv(A, xv, yv)
            outs.append(yv.array())
        truth = oracle.truth_csr(rp, col, vals, x, y0)
        assert rel_err(outs[0], truth) <= TOL[np.dtype(dt)], (name, storage, tiles)
        assert np.array_equal(outs[0].view(np.uint8), outs[1].view(np.uint8)), name
        empty = np.diff(rp) == 0
        assert np.array_equal(outs[0][empty].view(np.uint8), y0[empty].view(np.uint8)), name


@pytest.mark.parametrize("tile", [1024, 2048])
def test_csr_streamed_tile_kernel(gpu, oracle, tile):
    """Kernel 1 (bulk-copy streamed tiles of 1024 or 2048 nonzeros through a
    shared-memory ring), selected by the options struct."""
    from sciwasm.sparse_b200 import _lib
    for dt in DTYPES:
        for name, (rp, col, val) in _mats(dt).items():
            N = rp.size - 1
            x, y0 = _x_y(N, dt)
            A = gpu.csr_from_host(rp, col, val)
            A.opts = _lib.CsrOpts(1, 0, tile, 0)
            xv, yv = gpu.vec_from_host(x), gpu.vec_from_host(y0)
            gpu.spmv(A, xv, yv)
            err = rel_err(yv.array(), oracle.truth_csr(rp, col, val, x, y0))
            assert err <= TOL[np.dtype(dt)], (name, dt, err)
