"""The CUDA path against outputs of the reference's own JavaScript functions.

tests/golden/js_vectors.npz holds the inputs and outputs of SciWasm.Sparse's
host-side JavaScript -- coo_csr, coo_csc, num_cols/csr_ell,
num_diags/csr_dia, the level sets and the row reorderings -- executed from
their source by tests/golden/js_machine.py (see make_js_vectors.py).  The
device results must match them bit for bit, except where the reference's
shipped code leaves outputs unwritten (the reordered matrices' row
pointers) or stores the original order's row lengths; those are checked
against what they mean.
"""
import os

import numpy as np
import pytest

from test_js_vectors import case, same

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TAGS = ["f32", "f64"]


@pytest.fixture(scope="module")
def vec():
    return np.load(os.path.join(HERE, "golden", "js_vectors.npz"))


@pytest.mark.parametrize("tag", TAGS)
def test_coo_csr_and_coo_csc(gpu, vec, tag):
    c = case(vec, f"coo_csr_{tag}")
    A = gpu.coo_from_host(c["row"], c["col"], c["val"], int(c["N"]))
    C = gpu.coo_csr(A)
    assert same(C.row_array(), c["row_ptr"]) and same(C.col_array(), c["ccol"])
    assert same(C.val_array(), c["cval"])
    c = case(vec, f"coo_csc_{tag}")
    S = gpu.coo_csc(gpu.coo_from_host(c["row"], c["col"], c["val"], int(c["N"])))
    assert same(S.col_array(), c["col_ptr"]) and same(S.row_array(), c["srow"])
    assert same(S.val_array(), c["sval"])


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("name", ["band", "ragged"])
def test_csr_ell_and_csr_dia(gpu, vec, tag, name):
    c = case(vec, f"fmt_{name}_{tag}")
    A = gpu.csr_from_host(c["row_ptr"], c["col"], c["val"])
    assert gpu.num_cols(A) == int(c["nc"])
    assert gpu.num_diags(A) == [int(c["nd"]), int(c["stride"])]
    E = gpu.csr_ell(A)
    assert (E is not None) == bool(c["ell"])
    if E is not None:
        assert same(E.indices_array(), c["indices"]) and same(E.data_array(), c["edata"])
    D = gpu.csr_dia(A)
    assert (D is not None) == bool(c["dia"])
    if D is not None:
        assert same(D.offset_array(), c["offset"]) and same(D.data_array(), c["ddata"])


@pytest.mark.parametrize("name", ["lower", "narrow"])
def test_level_sets(gpu, vec, name):
    c = case(vec, f"levels_{name}")
    R = gpu.CSR_create_level_sets_with_reorder(gpu.csr_from_host(c["row_ptr"], c["col"], c["val"]))
    assert R.nlevels == int(c["nlevels"])
    assert same(R.level_index.to_host(), c["level_ptr"])
    assert same(R.permutation_index.to_host(), c["permutation"])
    assert same(R.row_array(), c["nrow_ptr"]) and same(R.col_array(), c["ncol"])
    assert same(R.val_array(), c["nval"])


@pytest.mark.parametrize("name", ["ragged", "band"])
def test_row_reordering(gpu, vec, name):
    c = case(vec, f"sortrows_{name}")
    A = gpu.csr_from_host(c["row_ptr"], c["col"], c["val"])
    assert gpu.calculate_csr_locality_index(A) == float(c["locality"])
    S = gpu.sort_rows_by_nnz(A)
    perm = c["permutation"]
    assert same(S.permutation_index.to_host(), perm)
    assert same(S.col_array(), c["ncol"]) and same(S.val_array(), c["nval"])
    assert [S.num_zero_rows, S.num_one_rows, S.num_two_rows, S.num_three_rows] == \
        c["small_rows"].tolist()
    # the reference leaves the row pointers unwritten and stores the original
    # order's lengths; the device writes the new matrix's own
    lens = c["nnz_per_row"][perm]
    assert same(S.nnz_row_index.to_host(), lens)
    assert same(S.row_array()[1:], np.cumsum(lens).astype(np.int32))
    yv = gpu.vec_from_host(c["y"])
    gpu.sort_y_rows_by_nnz(yv, S)
    assert same(yv.array(), c["y_new"])
    r = case(vec, f"reorder_nn_{name}")
    assert same(S.row_array(), r["srow_ptr"])
    R = gpu.reorder_NN(S, 16)
    assert same(R.permutation_index.to_host(), r["permutation"])
    assert same(R.col_array(), r["ncol"]) and same(R.val_array(), r["nval"])
