"""The CPU oracle against the hand-derived known-answer cases, plus
self-consistency properties of its restatement (CPU only)."""
import json
import os

import numpy as np
import pytest

from sciwasm.sparse_b200 import synth
from sciwasm.sparse_b200.sparse import fletcher_sum

KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                  "kat_reference_semantics.json")))


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_coo_csr_kat(oracle, dt):
    k = KAT["coo_csr_stable_duplicates"]
    rp, c, v = oracle.coo_csr(k["row"], k["col"], np.array(k["val"], dt), k["N"])
    assert rp.tolist() == k["row_ptr"]
    assert c.tolist() == k["csr_col"]
    assert v.tolist() == k["csr_val"]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_csr_dia_kat(oracle, dt):
    k = KAT["csr_dia_last_write_wins"]
    off, dat, nd, stride = oracle.csr_dia(k["row_ptr"], k["col"], np.array(k["val"], dt))
    assert (nd, stride) == (k["nd"], k["stride"])
    assert off.tolist() == k["offset"]
    assert dat.tolist() == k["data"]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_csr_ell_kat(oracle, dt):
    k = KAT["csr_ell_column_major"]
    ind, dat, nc = oracle.csr_ell(k["row_ptr"], k["col"], np.array(k["val"], dt))
    assert nc == k["nc"]
    assert ind.tolist() == k["indices"]
    assert dat.tolist() == k["data"]


def test_admission_kat(oracle):
    for c in KAT["admission"]["cases"]:
        assert oracle.format_admitted(c["w"], c["N"], c["nnz"]) == c["admitted"], c["why"]


def test_empty_matrix_refused(oracle):
    rp = np.zeros(5, np.int32)
    assert oracle.csr_ell(rp, np.zeros(0, np.int32), np.zeros(0, np.float32)) is None
    assert oracle.csr_dia(rp, np.zeros(0, np.int32), np.zeros(0, np.float32)) is None


def test_level_sets_kat(oracle):
    k = KAT["level_sets"]
    r = oracle.level_sets(k["row_ptr"], k["col"], np.array(k["val"], np.float64))
    assert r["nlevels"] == k["nlevels"]
    assert r["level"].tolist() == k["level"]
    assert r["level_ptr"].tolist() == k["level_ptr"]
    assert r["permutation"].tolist() == k["permutation"]
    assert r["order"].tolist() == k["order"]
    assert r["row_ptr"].tolist() == k["new_row_ptr"]
    assert r["col"].tolist() == k["new_col"]
    assert r["val"].tolist() == k["new_val"]


def test_level_sets_empty_row_kat(oracle):
    k = KAT["level_sets_empty_row"]
    r = oracle.level_sets(k["row_ptr"], k["col"], np.array(k["val"], np.float64))
    assert r["level"].tolist() == k["level"]
    assert r["nlevels"] == k["nlevels"]
    assert r["level_ptr"].tolist() == k["level_ptr"]
    assert r["permutation"].tolist() == k["permutation"]


@pytest.mark.parametrize("dt", [np.float32, np.float64])
def test_spts_kat(oracle, dt):
    k = KAT["spts_2x2"]
    args = (np.array(k["row_ptr"], np.int32), np.array(k["col"], np.int32),
            np.array(k["val"], dt), np.array(k["b"], dt))
    assert oracle.spts_csr(*args).tolist() == k["y"]
    assert oracle.spts_syncfree(*args).tolist() == k["y"]


def test_fletcher_kat(oracle):
    for c in KAT["fletcher"]["cases"]:
        assert oracle.fletcher(np.array(c["y"], np.float32)) == c["sum"]
        assert oracle.fletcher(np.array(c["y"], np.float64)) == c["sum"]
        assert fletcher_sum(c["y"]) == c["sum"]


def test_static_nnz_kat(oracle):
    k = KAT["static_nnz"]
    rs, re = oracle.static_nnz(k["row_ptr"], k["nw"])
    assert rs.tolist() == k["row_start"]
    assert re.tolist() == k["row_end"]


def test_empty_row_negative_zero_kat(oracle):
    k = KAT["csr_empty_row_keeps_negative_zero"]
    y0 = np.array(k["y0_bits_f32"], np.uint32).view(np.float32)
    x = np.array(k["x"], np.float32)
    y = oracle.spmv_csr(np.array(k["row_ptr"], np.int32), np.array(k["col"], np.int32),
                        np.array(k["val"], np.float32), x, y0)
    assert y.view(np.uint32).tolist() == np.array(k["csr_y"], np.float32).view(np.uint32).tolist()
    ye = oracle.spmv_ell(np.array(k["ell_indices"], np.int32), np.array(k["ell_data"], np.float32),
                         k["N"], k["ell_nc"], x, y0)
    assert ye.view(np.uint32).tolist() == np.array(k["ell_y"], np.float32).view(np.uint32).tolist()


# ----------------------------------------------------------- properties


def _random_coo(rng, N, nnz, dup=True):
    row = rng.integers(0, N, nnz).astype(np.int32)
    col = rng.integers(0, N, nnz).astype(np.int32)
    if dup and nnz > 4:
        row[-2:] = row[:2]
        col[-2:] = col[:2]
    return row, col


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_coo_csr_equals_stable_sort(oracle, seed):
    rng = np.random.default_rng(seed)
    N, nnz = 50, 400
    row, col = _random_coo(rng, N, nnz)
    val = rng.standard_normal(nnz)
    rp, c, v = oracle.coo_csr(row, col, val, N)
    order = np.lexsort((np.arange(nnz), col, row))  # stable by (row, col)
    assert np.array_equal(c, col[order])
    assert np.array_equal(v, val[order])
    assert np.array_equal(rp, np.concatenate([[0], np.cumsum(np.bincount(row, minlength=N))]))


def test_formats_agree_bitwise_on_sorted_csr(oracle):
    """DIA and ELL follow CSR's per-row order, so with finite x they give the
    same bits as CSR (the published checksums agree for ELL 1137/1137)."""
    rp, col, val = synth.banded(2000, half=3, seed=5, dtype=np.float32)
    x = synth.uniform_vec(2000, 7, dtype=np.float32)
    y0 = synth.uniform_vec(2000, 8, dtype=np.float32)
    ycsr = oracle.spmv_csr(rp, col, val, x, y0)
    off, dat, nd, stride = oracle.csr_dia(rp, col, val)
    ydia = oracle.spmv_dia(off, dat, 2000, x, y0)
    ind, edat, nc = oracle.csr_ell(rp, col, val)
    yell = oracle.spmv_ell(ind, edat, 2000, nc, x, y0)
    assert np.array_equal(ycsr.view(np.uint32), ydia.view(np.uint32))
    assert np.array_equal(ycsr.view(np.uint32), yell.view(np.uint32))


@pytest.mark.parametrize("nt", [1, 3, 5, 8])
def test_parallel_baseline_matches_serial(oracle, nt):
    rp, col, val = synth.power_law(3000, seed=9, dtype=np.float64, cap=300)
    x = synth.uniform_vec(3000, 1)
    y = np.zeros(3000)
    ys = oracle.spmv_csr(rp, col, val, x, y)
    yp = y.copy()
    oracle.par_spmv_csr(nt, rp, col, val, x, yp)
    assert np.array_equal(ys, yp)  # static_nnz keeps each row on one worker
    row = synth.csr_to_coo_rows(rp)
    yc = np.zeros(3000)
    wy = np.zeros(nt * 3000)
    oracle.par_spmv_coo(nt, row, col, val, x, yc, 3000, wy)
    assert np.max(np.abs(yc - ys)) < 1e-12


def test_level_solves_agree(oracle):
    rp, col, val = synth.random_lower(3000, seed=3)
    b = synth.uniform_vec(3000, 4)
    ls = oracle.level_sets(rp, col, val)
    truth = oracle.truth_spts(rp, col, val, b)
    y_row = oracle.spts_csr(rp, col, val, b)
    y_sf = oracle.spts_syncfree(rp, col, val, b)
    # level-ordered solve on the reordered matrix equals the row kernel in
    # natural order (rows of one level are independent)
    y_lv = oracle.spts_csr(ls["row_ptr"], ls["col"], ls["val"], b[ls["permutation"]])
    assert np.array_equal(y_lv, y_row[ls["permutation"]])
    for y in (y_row, y_sf):
        assert np.max(np.abs(y - truth) / np.maximum(np.abs(truth), 1e-300)) < 1e-12
    yp = np.zeros(3000)
    oracle.par_spts_level(5, ls["level_ptr"], ls["row_ptr"], ls["col"], ls["val"],
                          b[ls["permutation"]], yp)
    assert np.array_equal(yp, y_lv)


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("nt", [1, 3, 5, 8])
def test_parallel_syncfree_matches_serial(oracle, dt, nt):
    """The pthread sync-free baseline (cyclic rows, ready flags) gives the
    serial sync-free restatement's bits for any worker count."""
    for rp, col, val in (synth.random_lower(20_000, seed=5, band=300, dtype=dt),
                         synth.laplacian_3d_lower(12, dtype=dt)):
        N = rp.size - 1
        b = synth.uniform_vec(N, 6, dtype=dt)
        want = oracle.spts_syncfree(rp, col, val, b)
        y = np.full(N, np.nan, dt)
        oracle.par_spts_syncfree(nt, rp, col, val, b, y)
        assert np.array_equal(y.view(np.uint8), want.view(np.uint8))


def test_laplacian3d_levels(oracle):
    rp, col, val = synth.laplacian_3d_lower(16)
    ls = oracle.level_sets(rp, col, val)
    assert ls["nlevels"] == 3 * 15 + 1
    n = 16
    idx = np.arange(n ** 3)
    assert np.array_equal(ls["level"], idx // (n * n) + (idx // n) % n + idx % n)


def test_quick_sort_coo_sorts(oracle):
    rng = np.random.default_rng(4)
    row, col = _random_coo(rng, 40, 300)
    val = rng.standard_normal(300).astype(np.float32)
    r, c, v = oracle.quick_sort_coo(row, col, val)
    key = r.astype(np.int64) * 40 + c
    assert np.all(np.diff(key) >= 0)
    assert sorted(zip(row.tolist(), col.tolist(), val.tolist())) == \
        sorted(zip(r.tolist(), c.tolist(), v.tolist()))


def test_static_nnz_host_mirror_matches_oracle(oracle):
    from sciwasm.sparse_b200.sparse import static_nnz
    k = KAT["static_nnz"]
    rs, re = static_nnz(np.array(k["row_ptr"]), k["nw"])
    assert rs.tolist() == k["row_start"] and re.tolist() == k["row_end"]
    for seed, nw in [(0, 1), (1, 3), (2, 5), (3, 8), (4, 64)]:
        rp, col, val = synth.power_law(3000, seed=seed, cap=500)
        a = static_nnz(rp, nw)
        b = oracle.static_nnz(rp, nw)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (seed, nw)
    rp = np.array([0, 0, 0, 5, 5, 9], np.int32)  # empty rows
    for nw in (1, 2, 4, 7):
        a = static_nnz(rp, nw)
        b = oracle.static_nnz(rp, nw)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), nw
