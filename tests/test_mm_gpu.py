"""Matrix Market input on the device: the COO of create_COO_from_MM and
create_LCOO_from_MM is bit-identical to the oracle's (distinct coordinates,
so quick_sort_COO's order is the unique sorted order), in f32 and f64, and
the triangular matrix it builds solves like any other."""
import os

import numpy as np
import pytest

from conftest import rel_err
from test_mm import FILES, GOLD, KAT, _text, make_mm

pytestmark = pytest.mark.gpu


def _check(gpu, oracle, text, dtype, tmp_path=None):
    info = gpu.read_matrix_MM(text, nthreads=4)
    oinfo = oracle.mm_read(text)
    assert info.nnz == oinfo["nnz"]
    for lower, make in ((False, gpu.create_COO_from_MM), (True, gpu.create_LCOO_from_MM)):
        A = make(info, dtype)
        r, c, v = oracle.mm_coo(oinfo, dtype, lower=lower)
        assert A.N == oinfo["nrows"] and A.nnz == r.size
        assert np.array_equal(A.row_array(), r) and np.array_equal(A.col_array(), c)
        assert np.array_equal(A.val_array().view(np.uint8), v.view(np.uint8))
        # the Matrix Market COO is row-sorted: its SpMV takes the sorted-rows kernel
        assert A.rows_sorted
        if A.nnz:
            from conftest import TOL
            # x covers every column (files may have more columns than rows)
            nx = max(A.N, int(c.max()) + 1)
            x = np.random.default_rng(2).uniform(-1, 1, nx).astype(dtype)
            xv, yv = gpu.vec_from_host(x), gpu.create_vec(A.N, 0, dtype)
            gpu.spmv(A, xv, yv)
            rp = np.concatenate([[0], np.cumsum(np.bincount(r, minlength=A.N))]).astype(np.int32)
            truth = oracle.truth_csr(rp, c, v, x)
            assert rel_err(yv.array(), truth) <= TOL[np.dtype(dtype)]


@pytest.mark.parametrize("name", FILES)
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_kat_files(gpu, oracle, name, dtype):
    _check(gpu, oracle, _text(name), dtype)
    k = KAT[name]
    A = gpu.mmread(os.path.join(GOLD, "mm", name), dtype)  # the file path route
    assert A.row_array().tolist() == k["coo"]["row"]
    assert A.col_array().tolist() == k["coo"]["col"]
    assert np.array_equal(A.val_array(), np.array(k["coo"]["val"], dtype))


@pytest.mark.parametrize("field,sym", [("real", "general"), ("real", "symmetric"),
                                       ("integer", "general"), ("pattern", "symmetric")])
def test_generated_files(gpu, oracle, field, sym):
    rng = np.random.default_rng(11)
    _check(gpu, oracle, make_mm(rng, 2000, 2000, 40_000, field, sym), np.float32)
    _check(gpu, oracle, make_mm(rng, 1000, 1000, 9_000, field, sym), np.float64)


def test_lower_factor_solves(gpu, oracle):
    rng = np.random.default_rng(12)
    text = make_mm(rng, 3000, 3000, 20_000, "real", "symmetric")
    L = gpu.coo_csr(gpu.create_LCOO_from_MM(gpu.read_matrix_MM(text), np.float64))
    plan = gpu.SptsPlan(L)
    assert plan.solvable  # the unit diagonal is the last entry of every row
    b = rng.uniform(-1, 1, L.N)
    y = gpu.create_vec(L.N, 0, np.float64)
    gpu.spts(L, gpu.vec_from_host(b), y, algo="hybrid")
    truth = oracle.truth_spts(L.row_array(), L.col_array(), L.val_array(), b)
    assert rel_err(y.array(), truth) <= 1e-12


def test_empty_and_all_zero(gpu):
    text = b"%%MatrixMarket matrix coordinate real general\n5 5 0\n"
    info = gpu.read_matrix_MM(text)
    assert info.nnz == 0 and gpu.create_COO_from_MM(info).nnz == 0
    assert gpu.create_LCOO_from_MM(info).nnz == 5  # the unit diagonal alone
    text = b"%%MatrixMarket matrix coordinate real general\n3 3 2\n1 1 0\n2 3 0.0\n"
    assert gpu.create_COO_from_MM(gpu.read_matrix_MM(text)).nnz == 0
