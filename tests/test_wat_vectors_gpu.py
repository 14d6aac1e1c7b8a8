"""The CUDA path against outputs of the reference's own WebAssembly kernels.

The vectors in tests/golden/wat_vectors.npz were produced by executing
SciWasm.Sparse's .wat kernels (tests/golden/make_wat_vectors.py).  Results
that the device computes in the reference's order (DIA, ELL, the structure
kernels, the exact maps, reductions and every triangular solve) must match
bit for bit; CSR and COO SpMV add in a different order on the device and are
held to the SpMV tolerance against the same vectors.
"""
import os
import sys

import numpy as np
import pytest

from conftest import TOL, rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))

from make_wat_vectors import load_case  # noqa: E402
from test_wat_vectors import OPS, same  # noqa: E402

pytestmark = pytest.mark.gpu
TAGS = ["f32", "f64"]


@pytest.fixture(scope="module")
def vec():
    return np.load(os.path.join(HERE, "golden", "wat_vectors.npz"))


def _tol(a):
    return TOL[np.dtype(a.dtype)]


@pytest.mark.parametrize("tag", TAGS)
def test_spmv_formats(gpu, vec, tag):
    c = load_case(vec, f"spmv_csr_{tag}")
    A = gpu.csr_from_host(c["row_ptr"], c["col"], c["val"])
    yv = gpu.vec_from_host(c["y0"])
    gpu.spmv(A, gpu.vec_from_host(c["x"]), yv)
    assert rel_err(yv.array(), c["y"]) <= 2 * _tol(c["y"])
    empty = np.diff(c["row_ptr"]) == 0
    assert same(yv.array()[empty], c["y"][empty])
    c = load_case(vec, f"spmv_csr3_{tag}")
    yv = gpu.vec_from_host(c["y0"])
    gpu.spmv(A, gpu.vec_from_host(c["x"]), yv, inner_max=3)
    assert rel_err(yv.array(), c["y"]) <= 4 * _tol(c["y"])
    c = load_case(vec, f"spmv_coo_{tag}")
    C = gpu.coo_from_host(c["row"], c["col"], c["val"], int(c["N"]))
    yv = gpu.vec_from_host(c["y0"])
    gpu.spmv(C, gpu.vec_from_host(c["x"]), yv)
    assert rel_err(yv.array(), c["y"]) <= 2 * _tol(c["y"])
    c = load_case(vec, f"spmv_dia_{tag}")
    D = gpu.dia_from_host(c["offset"], c["data"], int(c["N"]))
    yv = gpu.vec_from_host(c["y0"])
    gpu.spmv(D, gpu.vec_from_host(c["x"]), yv)
    assert same(yv.array(), c["y"])
    c = load_case(vec, f"spmv_ell_{tag}")
    E = gpu.ell_from_host(c["indices"], c["data"], int(c["nc"]), int(c["N"]))
    yv = gpu.vec_from_host(c["y0"])
    gpu.spmv(E, gpu.vec_from_host(c["x"]), yv)
    assert same(yv.array(), c["y"])


def test_eliminate_zeros(gpu, vec):
    c = load_case(vec, "nz_coo_f32")
    Z = gpu.eliminate_zeros(gpu.coo_from_host(c["row"], c["col"], c["val"], 200))
    assert Z.nnz == int(c["count"])
    assert same(Z.row_array(), c["orow"]) and same(Z.col_array(), c["ocol"])
    assert same(Z.val_array(), c["oval"])
    c = load_case(vec, "nz_csr_f32")
    Z = gpu.eliminate_zeros(gpu.csr_from_host(c["row_ptr"], c["col"], c["val"]))
    assert same(Z.row_array(), c["orow_ptr"]) and same(Z.col_array(), c["ocol"])
    assert same(Z.val_array(), c["oval"])
    c = load_case(vec, "nz_dia_f32")
    Z = gpu.eliminate_zeros(gpu.dia_from_host(c["offset"], c["data"], int(c["N"]),
                                              nnz=c["data"].size))
    assert (Z.ndiags, Z.nnz) == (int(c["count_diags"]), int(c["count"]))
    assert same(Z.offset_array(), c["ooffset"]) and same(Z.data_array(), c["odata"])
    c = load_case(vec, "nz_ell_f32")
    Z = gpu.eliminate_zeros(gpu.ell_from_host(c["indices"], c["data"], int(c["nc"]), int(c["N"]),
                                              nnz=c["data"].size))
    assert (Z.ncols, Z.nnz) == (int(c["count_cols"]), int(c["count"]))
    assert same(Z.data_array(), c["odata"]) and same(Z.indices_array(), c["oindices"])


def test_transpose(gpu, vec):
    c = load_case(vec, "tr_csr_f32")
    T = gpu.transpose(gpu.csr_from_host(c["row_ptr"], c["col"], c["val"]))
    assert same(T.row_array(), c["orow_ptr"]) and same(T.col_array(), c["ocol"])
    assert same(T.val_array(), c["oval"])
    c = load_case(vec, "tr_dia_f32")
    T = gpu.transpose(gpu.dia_from_host(c["offset"], c["data"], int(c["N"])))
    assert same(T.offset_array(), c["ooffset"]) and same(T.data_array(), c["odata"])
    c = load_case(vec, "tr_ell_f32")
    T = gpu.transpose(gpu.ell_from_host(c["indices"], c["data"], int(c["nc"]), int(c["N"])))
    assert T.ncols == int(c["ncols"])
    assert same(T.data_array(), c["odata"]) and same(T.indices_array(), c["oindices"])


@pytest.mark.parametrize("tag", TAGS)
def test_reductions(gpu, vec, tag):
    for k in (0, 3, -4):
        c = load_case(vec, f"diag{k}_{tag}")
        A = gpu.coo_from_host(c["row"], c["col"], c["val"], int(c["N"]))
        assert same(A.diagonal(k).array(), c["diag"]), k
    c = load_case(vec, f"min_{tag}")
    A = gpu.coo_from_host(c["row"], c["col"], c["val"], int(c["N"]))
    assert same(A.min(1).array(), c["out"])


@pytest.mark.parametrize("tag", TAGS)
def test_spts_csc(gpu, vec, tag):
    cases = ["spts_csc4"] + (["spts_csc"] if tag == "f32" else [])
    for case in cases:
        c = load_case(vec, f"{case}_{tag}")
        n = c["col_ptr"].size - 1
        S = gpu.sparse_CSC_t(gpu.DeviceArray.from_host(c["col_ptr"]),
                             gpu.DeviceArray.from_host(c["row"]),
                             gpu.DeviceArray.from_host(c["val"]), n, c["row"].size)
        bv = gpu.vec_from_host(c["x"])
        y = gpu.create_vec(n, 0, c["val"].dtype)
        gpu.spts_csc(S, bv, y)
        assert same(y.array(), c["y"]), case


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("op", sorted(OPS))
def test_exact_maps(gpu, vec, tag, op):
    pi = np.float32(np.pi) if tag == "f32" else np.pi
    p = float(pi) if op in ("deg2rad", "rad2deg") else 0.0
    c = load_case(vec, f"map_{op}_coo_{tag}")
    n = c["val"].size
    idx = np.arange(n, dtype=np.int32)
    A = gpu.coo_from_host(idx, idx, c["val"], n)
    if "out" in c:
        assert same(gpu.map_copy(A, op, p).val_array(), c["out"])
    gpu.map_inplace(A, op, p)
    assert same(A.val_array(), c["self_out"])
    c = load_case(vec, f"map_{op}_ell_{tag}")
    rows = c["val"].size // 2
    E = gpu.ell_from_host(np.zeros(c["val"].size, np.int32), c["val"], 2, rows)
    assert same(gpu.map_copy(E, op, p).data_array(), c["out"])
    c = load_case(vec, f"map_{op}_dia_{tag}")
    D = gpu.dia_from_host(c["offset"], c["data"], int(c["N"]))
    if tag == "f32":
        assert same(gpu.map_copy(D, op, p).data_array(), c["out"])
    else:
        gpu.map_inplace(D, op, p)
        assert same(D.data_array(), c["out"])


@pytest.mark.parametrize("tag", TAGS)
def test_multiply_scalar(gpu, vec, tag):
    c = load_case(vec, f"map_multiply_coo_{tag}")
    n = c["val"].size
    idx = np.arange(n, dtype=np.int32)
    A = gpu.coo_from_host(idx, idx, c["val"], n)
    gpu.map_inplace(A, "multiply", float(c["p"]))
    assert same(A.val_array(), c["self_out"])


@pytest.mark.parametrize("name", ["lower", "lower_narrow"])
def test_spts(gpu, vec, name):
    c = load_case(vec, f"spts_syncfree_{name}")
    A = gpu.csr_from_host(c["row_ptr"], c["col"], c["val"])
    bv = gpu.vec_from_host(c["b"])
    y = gpu.create_vec(c["b"].size, 0, np.float32)
    gpu.spts(A, bv, y, algo="syncfree")
    assert same(y.array(), c["y"])
    # The reference's level solve ran on the level-ordered system P L P^T y' = b'.
    # The device solves L y = b in natural order: with b = P^T b', y = P^T y'.
    c = load_case(vec, f"spts_level_{name}")
    perm = c["permutation"]
    b = np.empty_like(c["b"])
    b[perm] = c["b"]
    A = gpu.csr_from_host(c["row_ptr"], c["col"], c["val"])
    bv = gpu.vec_from_host(b)
    hybrid = load_case(vec, f"spts_hybrid_{name}")
    for algo, want in (("level", c["y"]), ("hybrid", hybrid["y"])):
        y = gpu.create_vec(b.size, 0, np.float32)
        gpu.spts(A, bv, y, algo=algo)
        assert same(y.array()[perm], want), algo
