"""The oracle against outputs of the reference's own WebAssembly kernels.

tests/golden/wat_vectors.npz holds inputs and outputs of SciWasm.Sparse's
hand-written .wat kernels, executed by tests/golden/wat_machine.py (see
make_wat_vectors.py for how they were made).  Every comparison here is bit
for bit: the oracle restates those kernels and must give the same bits, which
pins it to the reference as it ships.
"""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_wat_vectors import load_case  # noqa: E402

OPS = {"sign": 7, "abs": 8, "neg": 9, "sqrt": 10, "ceil": 11, "floor": 12, "trunc": 13,
       "nearest": 14, "deg2rad": 5, "rad2deg": 6}
TAGS = ["f32", "f64"]


@pytest.fixture(scope="module")
def vec():
    return np.load(os.path.join(HERE, "golden", "wat_vectors.npz"))


def same(a, b):
    """Bit-identical, except that any NaN equals any NaN: WebAssembly leaves
    the sign and payload of a NaN result nondeterministic."""
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    if a.dtype.kind == "f":
        na, nb = np.isnan(a), np.isnan(b)
        if not np.array_equal(na, nb):
            return False
        a, b = a[~na], b[~nb]
    return np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("tag", TAGS)
def test_spmv(vec, oracle, tag):
    c = load_case(vec, f"spmv_csr_{tag}")
    assert same(oracle.spmv_csr(c["row_ptr"], c["col"], c["val"], c["x"], c["y0"]), c["y"])
    c = load_case(vec, f"spmv_csr3_{tag}")
    y = c["y0"]
    for _ in range(3):
        y = oracle.spmv_csr(c["row_ptr"], c["col"], c["val"], c["x"], y)
    assert same(y, c["y"])
    c = load_case(vec, f"spmv_coo_{tag}")
    assert same(oracle.spmv_coo(c["row"], c["col"], c["val"], c["x"], c["y0"]), c["y"])
    c = load_case(vec, f"spmv_dia_{tag}")
    assert same(oracle.spmv_dia(c["offset"], c["data"], int(c["N"]), c["x"], c["y0"],
                                int(c["stride"])), c["y"])
    c = load_case(vec, f"spmv_ell_{tag}")
    assert same(oracle.spmv_ell(c["indices"], c["data"], int(c["N"]), int(c["nc"]), c["x"], c["y0"]),
                c["y"])


@pytest.mark.parametrize("tag", TAGS)
def test_spmv_wrappers_inner_max(vec, oracle, tag):
    """The _wrapper exports repeat y += A x inner_max times."""
    c = load_case(vec, f"spmv_coo3_{tag}")
    y = c["y0"]
    for _ in range(3):
        y = oracle.spmv_coo(c["row"], c["col"], c["val"], c["x"], y)
    assert same(y, c["y"])
    c = load_case(vec, f"spmv_dia3_{tag}")
    y = c["y0"]
    for _ in range(3):
        y = oracle.spmv_dia(c["offset"], c["data"], int(c["N"]), c["x"], y, int(c["stride"]))
    assert same(y, c["y"])
    c = load_case(vec, f"spmv_ell3_{tag}")
    y = c["y0"]
    for _ in range(3):
        y = oracle.spmv_ell(c["indices"], c["data"], int(c["N"]), int(c["nc"]), c["x"], y)
    assert same(y, c["y"])


@pytest.mark.parametrize("tag", TAGS)
def test_sum_coo_as_shipped_is_not_a_row_sum(vec, oracle, tag):
    """The shipped sum_coo export advances its row counter for every entry it
    adds, so its output is not the row sums (no JS method calls it).  The
    library gives row sums (a deliberate difference); this records what the
    export does."""
    c = load_case(vec, f"sum_coo_{tag}")
    rows = oracle.sum_coo_rows(1, c["row"], c["val"], int(c["N"]))
    assert not same(rows, c["out"])


def test_eliminate_zeros(vec, oracle):
    c = load_case(vec, "nz_coo_f32")
    orow, ocol, oval = oracle.copy_nonzeros_coo(c["row"], c["col"], c["val"])
    assert orow.size == int(c["count"])
    assert same(orow, c["orow"]) and same(ocol, c["ocol"]) and same(oval, c["oval"])
    c = load_case(vec, "nz_csr_f32")
    orp, ocol, oval = oracle.copy_nonzeros_csr(c["row_ptr"], c["col"], c["val"])
    assert same(orp, c["orow_ptr"]) and same(ocol, c["ocol"]) and same(oval, c["oval"])
    c = load_case(vec, "nz_dia_f32")
    cd, cnt, ooff, odat = oracle.nonzeros_dia(c["offset"], c["data"], int(c["N"]), int(c["stride"]))
    assert (cd, cnt) == (int(c["count_diags"]), int(c["count"]))
    assert same(ooff, c["ooffset"]) and same(odat, c["odata"])
    c = load_case(vec, "nz_ell_f32")
    onc, cnt, od, oi = oracle.nonzeros_ell(c["data"], c["indices"], int(c["nc"]), int(c["N"]))
    assert (onc, cnt) == (int(c["count_cols"]), int(c["count"]))
    assert same(od, c["odata"]) and same(oi, c["oindices"])


def test_transpose(vec, oracle):
    c = load_case(vec, "tr_csr_f32")
    orp, ocol, oval = oracle.transpose_csr(c["row_ptr"], c["col"], c["val"])
    assert same(orp, c["orow_ptr"]) and same(ocol, c["ocol"]) and same(oval, c["oval"])
    c = load_case(vec, "tr_dia_f32")
    ooff, odat = oracle.transpose_dia(c["offset"], c["data"], int(c["N"]), int(c["stride"]))
    assert same(ooff, c["ooffset"]) and same(odat, c["odata"])
    c = load_case(vec, "tr_ell_f32")
    onc, od, oi = oracle.transpose_ell(c["data"], c["indices"], int(c["nc"]), int(c["N"]))
    assert onc == int(c["ncols"])
    assert same(od, c["odata"]) and same(oi, c["oindices"])


@pytest.mark.parametrize("tag", TAGS)
def test_reductions(vec, oracle, tag):
    for k in (0, 3, -4):
        c = load_case(vec, f"diag{k}_{tag}")
        assert same(oracle.diagonal_coo(k, c["row"], c["col"], c["val"], int(c["N"])), c["diag"]), k
    c = load_case(vec, f"min_{tag}")
    assert same(oracle.min_coo(1, c["row"], c["val"], int(c["N"])), c["out"])


@pytest.mark.parametrize("tag", TAGS)
def test_spts_csc(vec, oracle, tag):
    """Columns whose entries below the diagonal come in fours run only the
    kernel's 4-wide SIMD body: bit-identical in both precisions.  With a
    remainder, the FP64 module's scalar loop addresses y as row*4 bytes (a
    4-byte scale on 8-byte values, sparse_opt_64.wat spts_csc $inner_loop),
    so its output is not a triangular solve; the oracle keeps the FP32
    module's per-entry rule (row*4 on 4-byte values), which the FP64 SIMD body
    also follows, and matches the FP32 module bit for bit on every column."""
    c = load_case(vec, f"spts_csc4_{tag}")
    assert same(oracle.spts_csc(c["col_ptr"], c["row"], c["val"], c["x"]), c["y"])
    c = load_case(vec, f"spts_csc_{tag}")
    got = oracle.spts_csc(c["col_ptr"], c["row"], c["val"], c["x"])
    if tag == "f32":
        assert same(got, c["y"])
    else:
        assert not same(got, c["y"])


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("op", sorted(OPS))
def test_exact_maps(vec, oracle, tag, op):
    pi = np.float32(np.pi) if tag == "f32" else np.pi
    p = float(pi) if op in ("deg2rad", "rad2deg") else 0.0
    c = load_case(vec, f"map_{op}_coo_{tag}")
    want = oracle.map_values(c["val"], 0, OPS[op], p)
    if "out" in c:
        assert same(want, c["out"])
    assert same(want, c["self_out"])
    c = load_case(vec, f"map_{op}_ell_{tag}")
    assert same(oracle.map_values(c["val"], 1, OPS[op], p), c["out"])
    c = load_case(vec, f"map_{op}_dia_{tag}")
    got = oracle.map_dia(c["offset"], c["data"], int(c["N"]), OPS[op], p,
                         out=None if tag == "f32" else c["data"], stride=int(c["stride"]))
    assert same(got, c["out"])


@pytest.mark.parametrize("tag", TAGS)
def test_multiply_scalar(vec, oracle, tag):
    c = load_case(vec, f"map_multiply_coo_{tag}")
    assert same(oracle.map_values(c["val"], 0, 15, float(c["p"])), c["self_out"])


@pytest.mark.parametrize("name", ["lower", "lower_narrow"])
def test_spts(vec, oracle, name):
    c = load_case(vec, f"spts_syncfree_{name}")
    assert same(oracle.spts_syncfree(c["row_ptr"], c["col"], c["val"], c["b"]), c["y"])
    c = load_case(vec, f"spts_level_{name}")
    assert same(oracle.spts_csr(c["lrow_ptr"], c["lcol"], c["lval"], c["b"]), c["y"])
    L = oracle.level_sets(c["row_ptr"], c["col"], c["val"])
    assert same(L["row_ptr"], c["lrow_ptr"]) and same(L["col"], c["lcol"])
    # the reference's hybrid (level-ordered rows with sync-free waits) computes
    # each row as the level-set row kernel does
    c = load_case(vec, f"spts_hybrid_{name}")
    assert same(oracle.spts_csr(c["lrow_ptr"], c["lcol"], c["lval"], c["b"]), c["y"])
    # the SpTS module's own hybrid uses the sync-free row arithmetic instead
    # (subtract as you go): the reference ships both; the device's "hybrid"
    # is the first, its "syncfree" computes the second's values
    c = load_case(vec, f"spts_lsf_{name}")
    assert same(oracle.spts_syncfree(c["lrow_ptr"], c["lcol"], c["lval"], c["b"]), c["y"])
    assert not same(oracle.spts_csr(c["lrow_ptr"], c["lcol"], c["lval"], c["b"]), c["y"])
    # ... and the natural-order sync-free solve, permuted, gives the same bits
    lv = load_case(vec, f"spts_level_{name}")
    perm = lv["permutation"]
    b = np.empty_like(c["b"])
    b[perm] = c["b"]
    y = oracle.spts_syncfree(lv["row_ptr"], lv["col"], lv["val"], b)
    assert same(y[perm], c["y"])


def test_parallel_worker_kernels(vec, oracle):
    """The threaded CPU baseline (the oracle's port of the parallel build's
    worker partitioning) against the parallel build's own worker kernels run
    in turn: static_nnz row ranges for CSR, nnz ranges into private y copies
    summed in worker order for COO, even row ranges for DIA and ELL."""
    c = load_case(vec, "par_csr")
    nw = int(c["nw"])
    y = c["y0"].copy()
    oracle.par_spmv_csr(nw, c["row_ptr"], c["col"], c["val"], c["x"], y)
    assert same(y, c["y"])
    c = load_case(vec, "par_coo")
    y = c["y0"].copy()
    wy = np.zeros(nw * int(c["N"]), c["val"].dtype)
    oracle.par_spmv_coo(nw, c["row"], c["col"], c["val"], c["x"], y, int(c["N"]), wy)
    assert same(y, c["y"])
    # DIA and ELL: the column-layout worker kernels the port restates
    # (dia_col_basic, ell_col), and the row-layout ones (dia_row, ell_row),
    # whose per-row arithmetic is the same
    for case in ("par_dia_col", "par_dia"):
        c = load_case(vec, case)
        y = c["y0"].copy()
        oracle.par_spmv_dia(nw, c["offset"], c["data"], int(c["N"]), c["x"], y)
        assert same(y, c["y"]), case
    for case in ("par_ell_col", "par_ell"):
        c = load_case(vec, case)
        y = c["y0"].copy()
        oracle.par_spmv_ell(nw, c["indices"], c["data"], int(c["N"]), int(c["nc"]), c["x"], y)
        assert same(y, c["y"]), case
    # the row-layout kernels restated over row-by-row data (the vectors keep
    # the column layout; the reference's row kernels ran on its transpose)
    c = load_case(vec, "par_dia")
    N, nd = int(c["N"]), c["offset"].size
    y = c["y0"].copy()
    oracle.par_spmv_dia_rows(nw, c["offset"], c["data"].reshape(nd, N).T.copy(), N, c["x"], y)
    assert same(y, c["y"])
    c = load_case(vec, "par_ell")
    N, nc = int(c["N"]), int(c["nc"])
    y = c["y0"].copy()
    oracle.par_spmv_ell_rows(nw, c["indices"].reshape(nc, N).T.copy(),
                             c["data"].reshape(nc, N).T.copy(), N, nc, c["x"], y)
    assert same(y, c["y"])
