"""Format conversions on the GPU, bit-exact against the oracle and the
hand-derived known answers: coo_csr (sorted fast path and the radix-sort
path with duplicates), csr_ell and csr_dia with the reference's refusals."""
import json
import os

import numpy as np
import pytest

from sciwasm.sparse_b200 import synth

pytestmark = pytest.mark.gpu
KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                  "kat_reference_semantics.json")))


def bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint8)


def _same(a, b):
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(bits(a), bits(b))


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_coo_csr_kat(gpu, dt):
    k = KAT["coo_csr_stable_duplicates"]
    A = gpu.coo_from_host(k["row"], k["col"], np.array(k["val"], dt), k["N"])
    C = gpu.coo_csr(A)
    assert C.row_array().tolist() == k["row_ptr"]
    assert C.col_array().tolist() == k["csr_col"]
    assert C.val_array().tolist() == k["csr_val"]


def _random_coo(seed, N, nnz, dt, dup_frac=0.1):
    rng = np.random.default_rng(seed)
    row = rng.integers(0, N, nnz).astype(np.int32)
    col = rng.integers(0, N, nnz).astype(np.int32)
    nd = int(nnz * dup_frac)
    if nd:
        src = rng.integers(0, nnz, nd)
        dst = rng.integers(0, nnz, nd)
        row[dst], col[dst] = row[src], col[src]
    val = rng.standard_normal(nnz).astype(dt)
    return row, col, val


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("N,nnz", [(1, 5), (7, 40), (300, 5000), (70_000, 200_000),
                                   (3_000_000, 400_000)])
def test_coo_csr_unsorted_bitexact(gpu, oracle, dt, N, nnz):
    row, col, val = _random_coo(N + nnz, N, nnz, dt)
    want = oracle.coo_csr(row, col, val, N)
    C = gpu.coo_csr(gpu.coo_from_host(row, col, val, N))
    assert _same(C.row_array(), want[0])
    assert _same(C.col_array(), want[1])
    assert _same(C.val_array(), want[2])


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_coo_csr_sorted_fast_path(gpu, oracle, dt):
    rp, col, val = synth.banded(200_001, half=5, seed=3, dtype=dt)
    row = synth.csr_to_coo_rows(rp)
    # insert empty rows at the end and a duplicate pair
    N = 200_010
    row = np.concatenate([row, [N - 3, N - 3]]).astype(np.int32)
    col = np.concatenate([col, [5, 5]]).astype(np.int32)
    val = np.concatenate([val, np.array([1.5, -2.5], dt)])
    want = oracle.coo_csr(row, col, val, N)
    C = gpu.coo_csr(gpu.coo_from_host(row, col, val, N))
    assert _same(C.row_array(), want[0])
    assert _same(C.col_array(), want[1])
    assert _same(C.val_array(), want[2])


def test_coo_csr_powerlaw_shuffled(gpu, oracle):
    rp, col, val = synth.power_law(60_000, seed=5, dtype=np.float64, cap=2000, sort_cols=False)
    row = synth.csr_to_coo_rows(rp)
    perm = np.random.default_rng(0).permutation(row.size)
    row, col, val = row[perm], col[perm], val[perm]
    want = oracle.coo_csr(row, col, val, 60_000)
    C = gpu.coo_csr(gpu.coo_from_host(row, col, val, 60_000))
    assert _same(C.row_array(), want[0])
    assert _same(C.col_array(), want[1])
    assert _same(C.val_array(), want[2])


def _rows_of_lengths(lens, seed, dt, N=None):
    """A shuffled COO whose rows hold the given numbers of entries, with
    repeated columns (equal (row, col) keys), NaN and signed zeros."""
    rng = np.random.default_rng(seed)
    N = N or max(len(lens), max(lens) // 2 + 1)
    row = np.repeat(np.arange(len(lens), dtype=np.int32), lens)
    col = np.concatenate([rng.integers(0, max(1, l // 2 + 1), l) for l in lens]).astype(np.int32)
    col = np.minimum(col, N - 1)
    val = rng.standard_normal(row.size).astype(dt)
    val[rng.random(row.size) < 0.02] = np.nan
    val[rng.random(row.size) < 0.02] = -0.0
    perm = rng.permutation(row.size)
    return row[perm], col[perm], val[perm], N


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("longest", [2048, 5000])
def test_coo_csr_row_length_tiers(gpu, oracle, dt, longest):
    """Row lengths on both sides of every tier edge of the row-bucket sort
    (one thread up to 16, one warp up to 256, one block up to 2048); a row
    longer than 2048 sends the whole matrix through the radix sort.  Half the
    columns of a row repeat, so the tie order of equal keys is checked."""
    lens = [0, 1, 2, 3, 7, 8, 9, 15, 16, 17, 31, 32, 33, 255, 256, 257, 511, 512, 513, 1000,
            2047, longest, 0, 5]
    row, col, val, N = _rows_of_lengths(lens, longest, dt)
    want = oracle.coo_csr(row, col, val, N)
    C = gpu.coo_csr(gpu.coo_from_host(row, col, val, N))
    assert _same(C.row_array(), want[0])
    assert _same(C.col_array(), want[1])
    assert _same(C.val_array(), want[2])


def test_coo_csr_empty(gpu):
    A = gpu.coo_from_host(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32), 4)
    C = gpu.coo_csr(A)
    assert C.row_array().tolist() == [0, 0, 0, 0, 0]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_csr_ell_dia_kat(gpu, dt):
    k = KAT["csr_ell_column_major"]
    A = gpu.csr_from_host(k["row_ptr"], k["col"], np.array(k["val"], dt))
    assert gpu.num_cols(A) == k["nc"]
    E = gpu.csr_ell(A)
    assert E.ncols == k["nc"]
    assert E.indices_array().tolist() == k["indices"]
    assert E.data_array().tolist() == k["data"]
    kd = KAT["csr_dia_last_write_wins"]
    assert gpu.num_diags(A) == [kd["nd"], kd["stride"]]
    D = gpu.csr_dia(A)
    assert D.offset_array().tolist() == kd["offset"]
    assert D.data_array().tolist() == kd["data"]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", ["banded", "laplacian", "random_dups", "ragged"])
def test_csr_ell_dia_bitexact(gpu, oracle, dt, name):
    if name == "banded":
        rp, col, val = synth.banded(100_000, half=5, seed=1, dtype=dt)
    elif name == "laplacian":
        rp, col, val = synth.laplacian_2d(128, dtype=dt)
    elif name == "random_dups":
        row, c0, v0 = _random_coo(9, 3000, 12_000, dt, dup_frac=0.2)
        # keep entries within a band so DIA is admitted, duplicates included
        c0 = np.clip(row + (c0 % 7) - 3, 0, 2999).astype(np.int32)
        rp, col, val = oracle.coo_csr(row, c0, v0, 3000)
    else:
        rng = np.random.default_rng(2)
        lens = rng.integers(0, 4, 5000)
        lens[100] = 9
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
        rows = np.repeat(np.arange(5000), lens)
        col = np.clip(rows + rng.integers(-2, 3, rows.size), 0, 4999).astype(np.int32)
        val = rng.standard_normal(col.size).astype(dt)
    A = gpu.csr_from_host(rp, col, val)
    want = oracle.csr_ell(rp, col, val)
    E = gpu.csr_ell(A)
    if want is None:
        assert E is None
    else:
        assert E.ncols == want[2]
        assert _same(E.indices_array(), want[0])
        assert _same(E.data_array(), want[1])
    want = oracle.csr_dia(rp, col, val)
    D = gpu.csr_dia(A)
    if want is None:
        assert D is None
    else:
        assert (D.ndiags, D.stride) == (want[2], want[3])
        assert _same(D.offset_array(), want[0])
        assert _same(D.data_array(), want[1])


def test_refusals(gpu, oracle):
    rp, col, val = synth.power_law(30_000, seed=2, cap=2000)
    A = gpu.csr_from_host(rp, col, val)
    assert oracle.csr_ell(rp, col, val) is None and gpu.csr_ell(A) is None
    assert oracle.csr_dia(rp, col, val) is None and gpu.csr_dia(A) is None
    Z = gpu.csr_from_host(np.zeros(6, np.int32), np.zeros(0, np.int32), np.zeros(0))
    assert gpu.csr_ell(Z) is None and gpu.csr_dia(Z) is None


def test_convert_then_spmv_all_formats(gpu, oracle):
    """COO -> CSR -> DIA/ELL on the device, then SpMV in all four formats."""
    rp, col, val = synth.banded(50_000, half=5, seed=4)
    row = synth.csr_to_coo_rows(rp)
    x = synth.uniform_vec(50_000, 1)
    truth = oracle.truth_csr(rp, col, val, x)
    Acoo = gpu.coo_from_host(row, col, val, 50_000)
    Acsr = gpu.coo_csr(Acoo)
    for A in (Acoo, Acsr, gpu.csr_dia(Acsr), gpu.csr_ell(Acsr)):
        xv, yv = gpu.vec_from_host(x), gpu.create_vec(50_000, 0, np.float64)
        gpu.spmv(A, xv, yv)
        y = yv.array()
        assert np.max(np.abs(y - truth)) / np.max(np.abs(truth)) < 1e-12
