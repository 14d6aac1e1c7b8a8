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


@pytest.mark.parametrize("storage", ["f32", "f64", "bf16"])
def test_csr_block_stream_kernel(gpu, oracle, storage):
    """Kernel 3 (a warp per 32-row block streaming its nonzeros in 256-entry
    chunks): within the tolerance of the exact result on regular, skewed,
    ragged and empty-row matrices, rows without entries keep their bits, two
    runs give identical bits, and a col/val pair that is not 16-byte aligned
    takes the scalar-load form with the same result."""
    from sciwasm.sparse_b200 import _lib
    dt = np.float64 if storage == "f64" else np.float32
    mats = _mats(dt)
    mats["rows_over_blocks"] = synth.power_law(9_000, seed=8, dtype=dt, cap=3000, shift=0)
    for name, (rp, col, val) in mats.items():
        N = rp.size - 1
        x, y0 = _x_y(N, dt)
        A = gpu.csr_from_host(rp, col, val)
        vals = val
        if storage == "bf16":
            A = gpu.csr_with_storage(A, "bf16")
            vals = (A.val_array().astype(np.uint32) << 16).view(np.float32)
        A.opts = _lib.CsrOpts(3, 0, 0, 0)
        outs = []
        for _ in range(2):
            xv, yv = gpu.vec_from_host(x), gpu.vec_from_host(y0)
            gpu.spmv(A, xv, yv)
            outs.append(yv.array())
        truth = oracle.truth_csr(rp, col, vals, x, y0)
        assert rel_err(outs[0], truth) <= TOL[np.dtype(dt)], (name, storage)
        assert np.array_equal(outs[0].view(np.uint8), outs[1].view(np.uint8)), name
        empty = np.diff(rp) == 0
        assert np.array_equal(outs[0][empty].view(np.uint8), y0[empty].view(np.uint8)), name
        if storage != "bf16" and col.size > 1:
            # col/val one element into a buffer: 4-byte (f32) or 8-byte (f64)
            # aligned, not 16: the scalar-load form
            from sciwasm.sparse_b200.sparse import DeviceArray
            cbuf = DeviceArray.from_host(np.concatenate([[0], col]).astype(np.int32))
            vbuf = DeviceArray.from_host(np.concatenate([[0], val]).astype(dt))
            rpd = DeviceArray.from_host(rp)
            xv, yv = gpu.vec_from_host(x), gpu.vec_from_host(y0)
            code = _lib.SB_F64 if dt == np.float64 else _lib.SB_F32
            _lib.call("sb_spmv_csr_ex", code, rpd.ptr, cbuf.ptr + 4, vbuf.ptr + dt().itemsize,
                      xv.vec_index.ptr, yv.vec_index.ptr, N, col.size, 1,
                      __import__("ctypes").byref(A.opts), None)
            assert rel_err(yv.array(), truth) <= TOL[np.dtype(dt)], (name, "unaligned")


@pytest.mark.parametrize("dt", DTYPES)
def test_gather_dot_is_the_sum_of_the_product(gpu, oracle, dt):
    import ctypes
    from sciwasm.sparse_b200 import _lib
    from sciwasm.sparse_b200.sparse import DeviceArray
    for name in ("powerlaw", "ragged", "single"):
        rp, col, val = _mats(dt)[name]
        N = rp.size - 1
        x, _ = _x_y(N, dt)
        truth = float(np.sum(oracle.truth_csr(rp, col, val, x)))
        out = DeviceArray.from_host(np.zeros(1))
        c, v, xd = DeviceArray.from_host(col), DeviceArray.from_host(val), \
            DeviceArray.from_host(x)
        code = _lib.SB_F64 if dt == np.float64 else _lib.SB_F32
        _lib.call("sb_gather_dot", code, c.ptr, v.ptr, xd.ptr, col.size, out.ptr, None)
        got = float(out.to_host()[0])
        scale = float(np.sum(np.abs(val.astype(np.float64) * x[col])))
        assert abs(got - truth) <= 10 * TOL[np.dtype(dt)] * max(scale, 1e-300), name


def test_spmv_autotune_picks_dia_for_banded_and_keeps_parity(gpu, oracle):
    """The format autotuner: on a banded matrix (11 diagonals, 2M rows, FP64)
    DIA moves the fewest bytes and is chosen; the power-law matrix's DIA and
    ELL forms are refused by the admission test and never timed; the chosen
    object computes y <- y + A x within tolerance (DIA bit-identical to the
    oracle's serial loop)."""
    rp, col, val = synth.banded(2_000_000, half=5, seed=1, dtype=np.float64)
    N = rp.size - 1
    A = gpu.csr_from_host(rp, col, val)
    x, y0 = _x_y(N, np.float64)
    xv = gpu.vec_from_host(x)
    M, info = gpu.spmv_autotune(A, xv)
    assert info["dia_admitted"] and info["ndiags"] == 11 and info["ncols"] == 11
    assert info["bytes"]["dia"] < info["bytes"]["ell"] < info["bytes"]["csr"]
    assert info["format"] == "dia", info
    assert isinstance(M, gpu.sparse_DIA_t) and info["ms"]["dia"] < info["ms"]["csr"]
    yv = gpu.vec_from_host(y0)
    gpu.spmv(M, xv, yv)
    off, dat = synth.csr_to_dia_host(rp, col, val)
    assert np.array_equal(yv.array().view(np.uint8),
                          oracle.spmv_dia(off, dat, N, x, y0).view(np.uint8))
    del A, M
    rp, col, val = synth.power_law(200_000, seed=2, dtype=np.float64)
    N = rp.size - 1
    A = gpu.csr_from_host(rp, col, val)
    x, y0 = _x_y(N, np.float64)
    xv = gpu.vec_from_host(x)
    M, info = gpu.spmv_autotune(A, xv)
    assert not info["dia_admitted"] and not info["ell_admitted"]
    assert info["ms"]["dia"] is None and info["ms"]["ell"] is None
    assert info["format"] in ("csr", "coo") and info["ms"]["csr"] > 0
    yv = gpu.vec_from_host(y0)
    gpu.spmv(M, xv, yv)
    assert rel_err(yv.array(), oracle.truth_csr(rp, col, val, x, y0)) <= 1e-12


def _poisson_rows(N, mean, seed):
    """Poisson(mean) distinct uniform columns per row plus the diagonal."""
    rng = np.random.default_rng(seed)
    lens = rng.poisson(mean, N).astype(np.int64)
    cols = synth._distinct_uniform_cols(rng, lens, np.zeros(N, np.int64), np.full(N, N, np.int64))
    rows = np.repeat(np.arange(N), lens)
    allr = np.concatenate([rows, np.arange(N)])
    allc = np.concatenate([cols, np.arange(N)])
    key = np.unique(allr * N + allc)
    r, c = key // N, key % N
    rp = np.concatenate([[0], np.cumsum(np.bincount(r, minlength=N))]).astype(np.int32)
    return rp, c.astype(np.int32), rng.uniform(-1, 1, c.size).astype(np.float32)


def test_spmv_autotune_statistics_mode(gpu, oracle):
    """Without timing, the admitted format with the fewest compulsory bytes:
    DIA for banded and 5-point matrices, CSR row blocks for Poisson row
    lengths and, one warp per block, for skewed power-law rows, ELL for rows
    of one length (no row_ptr to read); the chosen object keeps parity."""
    cases = {"banded": (synth.banded(50_000, half=5, seed=1, dtype=np.float32), "dia", None),
             "lap2d": (synth.laplacian_2d(200, dtype=np.float32), "dia", None),
             "powerlaw": (synth.power_law(60_000, seed=2, dtype=np.float32), "csr", (0, 8, 1)),
             "poisson": (_poisson_rows(60_000, 12.0, seed=3), "csr", (0, 4, 0)),
             "uniform13": (synth.random_lower(60_000, per_row=12, band=60_000, seed=3,
                                              dtype=np.float32), "ell", None)}
    for name, ((rp, col, val), fmt, kernel) in cases.items():
        N = rp.size - 1
        A = gpu.csr_from_host(rp, col, val)
        M, info = gpu.spmv_autotune(A, timed=False)
        assert info["format"] == fmt, (name, info)
        assert all(v is None for v in info["ms"].values())
        if kernel is not None:
            o = info["csr_opts"]
            assert (o["kernel"], o["lanes_per_row"], o["grid"]) == kernel, (name, info)
        x, y0 = _x_y(N, np.float32)
        yv = gpu.vec_from_host(y0)
        gpu.spmv(M, gpu.vec_from_host(x), yv)
        assert rel_err(yv.array(), oracle.truth_csr(rp, col, val, x, y0)) <= 1e-5, name


@pytest.mark.parametrize("shape", ["laplacian_even", "laplacian_odd", "band_even", "band_2mod4"])
def test_dia_bf16_storage(gpu, oracle, shape):
    """DIA with BF16 data (f32 x, y and sums): within tolerance of the FP64
    product of the stored values, and bit-identical to the batched DIA item
    on the same data (the same per-row order).  Even N takes two rows per
    thread, N a multiple of 4 four (offsets odd, even and multiples of 4:
    scalar, paired and quadruple x loads; edge groups per row), odd N one
    row per thread."""
    if shape == "laplacian_even":
        rp, col, val = synth.laplacian_2d(300, dtype=np.float32)
    elif shape == "laplacian_odd":
        rp, col, val = synth.laplacian_2d(301, dtype=np.float32)
    elif shape == "band_even":
        rp, col, val = synth.banded(20_000, half=5, seed=4, dtype=np.float32)
    else:
        rp, col, val = synth.banded(20_002, half=5, seed=4, dtype=np.float32)
    N = rp.size - 1
    D = gpu.csr_dia(gpu.csr_from_host(rp, col, val))
    Db = gpu.with_storage(D, "bf16")
    x, y0 = _x_y(N, np.float32)
    yv = gpu.vec_from_host(y0)
    gpu.spmv(Db, gpu.vec_from_host(x), yv)
    vb = (gpu.csr_with_storage(gpu.csr_from_host(rp, col, val), "bf16").val_array()
          .astype(np.uint32) << 16).view(np.float32)
    truth = oracle.truth_csr(rp, col, vb.astype(np.float64), x.astype(np.float64), y0)
    assert rel_err(yv.array(), truth) <= 1e-5
    ex = gpu.BatchExecutor("bf16", capacity=2)
    xd, yd = gpu.DeviceArray.from_host(x), gpu.DeviceArray.from_host(y0)
    ex.run([(Db, xd, yd, 1)])
    gpu.synchronize()
    assert np.array_equal(yd.to_host().view(np.uint32), yv.array().view(np.uint32))


def test_clear_vec_and_init_x(gpu):
    """clear_vec / init_x (src/sequential/src/sparse32.js:1313-1322) on the device."""
    for dt in DTYPES:
        v = gpu.vec_from_host(np.full(1000, 3.5, dt))
        gpu.clear_vec(v)
        assert np.array_equal(v.array(), np.zeros(1000, dt))
        gpu.init_x(v)
        assert np.array_equal(v.array(), np.arange(1000, dtype=dt))
