"""The oracle against outputs of the reference's own JavaScript functions.

tests/golden/js_vectors.npz holds inputs and outputs of SciWasm.Sparse's
host-side JavaScript (coo_csr, coo_csc, quick_sort_COO, num_cols/csr_ell,
num_diags/csr_dia, static_nnz, CSR_create_level_sets_with_reorder), executed
by tests/golden/js_machine.py (see make_js_vectors.py).  Every comparison is
bit for bit.  The device conversions and level sets are checked bit for bit
against the same oracle functions by the -m gpu tests, at small and at full
size.
"""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
TAGS = ["f32", "f64"]


@pytest.fixture(scope="module")
def vec():
    return np.load(os.path.join(HERE, "golden", "js_vectors.npz"))


def case(z, name):
    pre = name + "/"
    return {k[len(pre):]: z[k] for k in z.files if k.startswith(pre)}


def same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.shape == b.shape and a.dtype == b.dtype and np.array_equal(
        a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("tag", TAGS)
def test_coo_csr(vec, oracle, tag):
    """Stable order of repeated (row, col) keys: the per-row bubble sort."""
    c = case(vec, f"coo_csr_{tag}")
    rp, col, val = oracle.coo_csr(c["row"], c["col"], c["val"], int(c["N"]))
    assert same(rp, c["row_ptr"]) and same(col, c["ccol"]) and same(val, c["cval"])


@pytest.mark.parametrize("tag", TAGS)
def test_coo_csc(vec, oracle, tag):
    c = case(vec, f"coo_csc_{tag}")
    cp, row, val = oracle.coo_csc(c["row"], c["col"], c["val"], int(c["N"]))
    assert same(cp, c["col_ptr"]) and same(row, c["srow"]) and same(val, c["sval"])


@pytest.mark.parametrize("tag", TAGS)
def test_quick_sort_coo(vec, oracle, tag):
    """The unstable quicksort, repeated keys included: the same pivots and
    swaps leave equal keys in the same order."""
    c = case(vec, f"qsort_{tag}")
    row, col, val = oracle.quick_sort_coo(c["row"], c["col"], c["val"])
    assert same(row, c["srow"]) and same(col, c["scol"]) and same(val, c["sval"])


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("name", ["band", "ragged"])
def test_csr_ell_and_csr_dia(vec, oracle, tag, name):
    c = case(vec, f"fmt_{name}_{tag}")
    rp, col, val = c["row_ptr"], c["col"], c["val"]
    assert oracle.num_cols(rp) == int(c["nc"])
    nd, stride = oracle.num_diags(rp, col)
    assert (nd, stride) == (int(c["nd"]), int(c["stride"]))
    ell = oracle.csr_ell(rp, col, val)
    assert (ell is not None) == bool(c["ell"])
    if ell is not None:
        assert same(ell[0], c["indices"]) and same(ell[1], c["edata"])
    dia = oracle.csr_dia(rp, col, val)
    assert (dia is not None) == bool(c["dia"])
    if dia is not None:
        assert same(dia[0], c["offset"]) and same(dia[1], c["ddata"])


def test_admission_outcomes_cover_both_branches(vec):
    assert bool(case(vec, "fmt_band_f32")["dia"]) and bool(case(vec, "fmt_band_f32")["ell"])
    assert not bool(case(vec, "fmt_ragged_f32")["dia"])


@pytest.mark.parametrize("name", ["static_nnz_200_3", "static_nnz_97_5", "static_nnz_6_8"])
def test_static_nnz(vec, oracle, name):
    c = case(vec, name)
    rs, re = oracle.static_nnz(c["row_ptr"], int(c["nw"]))
    assert same(rs, c["row_start"]) and same(re, c["row_end"])


@pytest.mark.parametrize("name", ["lower", "narrow", "empty_rows"])
def test_level_sets(vec, oracle, name):
    c = case(vec, f"levels_plain_{name}")
    L = oracle.level_sets(c["row_ptr"], c["col"], c["val"])
    assert L["nlevels"] == int(c["nlevels"])
    assert same(L["level_ptr"], c["level_ptr"]) and same(L["permutation"], c["permutation"])
    for kind in ("levels", "levels_spts"):     # sparse32.js's and spts32.js's copies
        c = case(vec, f"{kind}_{name}")
        L = oracle.level_sets(c["row_ptr"], c["col"], c["val"])
        assert L["nlevels"] == int(c["nlevels"])
        assert same(L["level_ptr"], c["level_ptr"])
        assert same(L["permutation"], c["permutation"])
        assert same(L["row_ptr"], c["nrow_ptr"]) and same(L["col"], c["ncol"])
        assert same(L["val"], c["nval"])
    c = case(vec, f"levels_{name}")
    L = oracle.level_sets(c["row_ptr"], c["col"], c["val"])
    assert L["nlevels"] == int(c["nlevels"])
    assert same(L["level_ptr"], c["level_ptr"])
    assert same(L["permutation"], c["permutation"])
    assert same(L["row_ptr"], c["nrow_ptr"]) and same(L["col"], c["ncol"])
    assert same(L["val"], c["nval"])


MM_CASES = ["gen_integer", "gen_pattern", "sym_pattern", "sym_real", "gen_real_seeded",
            "sym_real_seeded"]


@pytest.mark.parametrize("name", MM_CASES)
@pytest.mark.parametrize("lower", [False, True])
def test_matrix_market(vec, oracle, name, lower):
    """read_matrix_MM_files on load_file's lines, then create_COO_from_MM or
    create_LCOO_from_MM and quick_sort_COO: the oracle's reader and COO
    builder give the same nnz and the same (row, col, value) order."""
    c = case(vec, f"mm_{name}_{'lower' if lower else 'full'}")
    info = oracle.mm_read(c["text"].tobytes())
    assert info["nnz"] == int(c["nnz"])
    row, col, val = oracle.mm_coo(info, np.float32, lower=lower)
    assert same(row, c["row"]) and same(col, c["col"]) and same(val, c["val"])


@pytest.mark.parametrize("name", ["ragged", "band", "ragged_f64", "band_f64"])
def test_row_reordering(vec, oracle, name):
    """sort_rows_by_nnz, sort_y_rows_by_nnz and calculate_csr_locality_index
    as the parallel build ships them.  Its new matrix comes from a
    sparse_CSR_t without `nrows`, so the view it writes row pointers through
    is empty: the reference leaves them unwritten, the oracle (and the device)
    write the prefix sums of the row lengths."""
    c = case(vec, f"sortrows_{name}")
    assert oracle.csr_locality_index(c["row_ptr"], c["col"]) == float(c["locality"])
    S = oracle.sort_rows_by_nnz(c["row_ptr"], c["col"], c["val"])
    assert same(S["permutation"], c["permutation"])
    # the reference stores the original order's row lengths in the new
    # matrix's nnz_per_row; the oracle stores the new matrix's own
    assert same(c["nnz_per_row"], np.diff(c["row_ptr"]).astype(np.int32))
    assert same(S["nnz_per_row"], c["nnz_per_row"][c["permutation"]])
    assert same(S["col"], c["ncol"]) and same(S["val"], c["nval"])
    assert same(S["small_rows"], c["small_rows"])
    assert not np.any(c["nrow_ptr"])
    assert same(S["row_ptr"][1:], np.cumsum(S["nnz_per_row"]).astype(np.int32))
    assert same(oracle.unpermute_rows(c["permutation"], c["y"]), c["y_new"])


@pytest.mark.parametrize("name", ["ragged", "band", "ragged_f64", "band_f64"])
def test_reorder_nn(vec, oracle, name):
    """reorder_NN (w = 16) on the row-sorted matrix: the nearest-neighbour
    walk composed with the sort's permutation, and the reordered columns and
    values."""
    c = case(vec, f"reorder_nn_{name}")
    # the FP32 build keeps the similarity list in a Float32Array, the FP64
    # build (sparse64.js) in a Float64Array
    lb = 8 if name.endswith("_f64") else 4
    R = oracle.reorder_nn(c["srow_ptr"], c["scol"], c["sval"], w=16, perm_in=c["sperm"],
                          list_bytes=lb)
    assert same(R["permutation"], c["permutation"])
    assert same(R["col"], c["ncol"]) and same(R["val"], c["nval"])


def test_reorder_nn_list_precision_matters(vec, oracle):
    """On this matrix the FP64 build's double list walks differently from the
    float32 list that the FP32 build, the oracle's default and the device use
    for both precisions (a known difference for FP64 matrices)."""
    c = case(vec, "reorder_nn_ragged_f64")
    R = oracle.reorder_nn(c["srow_ptr"], c["scol"], c["sval"], w=16, perm_in=c["sperm"])
    assert not same(R["permutation"], c["permutation"])


@pytest.mark.parametrize("name", ["static_nnz_200_3", "static_nnz_97_5", "static_nnz_6_8"])
def test_static_nnz_host_partitioner(vec, name):
    """The library's own host partitioner (row shards across GPUs) gives the
    reference's ranges, including the row_end it leaves at 0."""
    from sciwasm.sparse_b200.sparse import static_nnz
    c = case(vec, name)
    rs, re = static_nnz(c["row_ptr"], int(c["nw"]))
    assert same(rs, c["row_start"]) and same(re, c["row_end"])


@pytest.mark.parametrize("i", [0, 1, 2])
def test_fletcher_sum(vec, oracle, i):
    """fletcher_sum_y, the checksum the reference benchmark prints for y:
    the oracle's and the library's host restatement give the same integer."""
    from sciwasm.sparse_b200.sparse import fletcher_sum
    c = case(vec, f"fletcher_{i}")
    assert oracle.fletcher(c["y"]) == int(c["sum"])
    assert fletcher_sum(c["y"]) == int(c["sum"])
