"""Level sets and triangular solves on the GPU: levels, level_ptr,
permutation, order and the reordered CSR bit-exact against the oracle (and
the hand-derived known answers); solves bit-identical to the oracle's
restatement of each reference kernel, and within tolerance of the
extended-precision truth; bounded waits report a timeout instead of hanging."""
import json
import os

import numpy as np
import pytest

from conftest import TOL
from sciwasm.sparse_b200 import SparseError, synth

pytestmark = pytest.mark.gpu
KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                  "kat_reference_semantics.json")))


def _ub(a):
    return np.ascontiguousarray(a).view(np.uint8)


def _check_levels(gpu, oracle, rp, col, val):
    want = oracle.level_sets(rp, col, val)
    A = gpu.csr_from_host(rp, col, val)
    R = gpu.CSR_create_level_sets_with_reorder(A)
    assert R.nlevels == want["nlevels"]
    assert np.array_equal(R.level_per_row.to_host(), want["level"])
    assert np.array_equal(R.level_index.to_host(), want["level_ptr"])
    assert np.array_equal(R.permutation_index.to_host(), want["permutation"])
    assert np.array_equal(R.order_index.to_host(), want["order"])
    assert np.array_equal(R.row_array(), want["row_ptr"])
    assert np.array_equal(R.col_array(), want["col"])
    assert np.array_equal(_ub(R.val_array()), _ub(want["val"]))
    return A


def test_level_sets_kat(gpu, oracle):
    k = KAT["level_sets"]
    _check_levels(gpu, oracle, np.array(k["row_ptr"], np.int32), np.array(k["col"], np.int32),
                  np.array(k["val"], np.float64))
    k = KAT["level_sets_empty_row"]
    A = gpu.csr_from_host(k["row_ptr"], k["col"], np.array(k["val"], np.float64))
    gpu.CSR_create_level_sets(A)
    assert A.level_per_row.to_host().tolist() == k["level"]
    assert A.level_index.to_host().tolist() == k["level_ptr"]
    assert A.permutation_index.to_host().tolist() == k["permutation"]
    assert not A._plan.solvable


@pytest.mark.parametrize("name", ["lap3d", "random_lower", "chain", "wide"])
def test_level_sets_bitexact(gpu, oracle, name):
    if name == "lap3d":
        rp, col, val = synth.laplacian_3d_lower(20)
    elif name == "random_lower":
        rp, col, val = synth.random_lower(60_000, seed=3, band=500)
    elif name == "chain":  # one level per row: the longest dependency chain
        N = 3000
        rp = np.arange(0, 2 * N, 2, dtype=np.int32)
        rp = np.concatenate([[0], np.arange(1, 2 * N - 1, 2), [2 * N - 1]]).astype(np.int32)
        col = np.concatenate([[0]] + [[i - 1, i] for i in range(1, N)]).astype(np.int32)
        val = np.ones(col.size)
    else:  # many rows at level 0 and 1
        N = 40_000
        rp = np.concatenate([[0], np.arange(1, N + 1)]).astype(np.int32)
        col = np.arange(N, dtype=np.int32)
        val = np.full(N, 2.0)
    _check_levels(gpu, oracle, rp, col, val)


def _chain(n, dt):
    """Lower bidiagonal: one row per level (a barrier per row in the level solve)."""
    rp = np.concatenate([[0], np.cumsum([1] + [2] * (n - 1))]).astype(np.int32)
    col = np.empty(rp[-1], np.int32)
    val = np.empty(rp[-1], dt)
    col[0], val[0] = 0, 2.0
    i = np.arange(1, n)
    col[rp[1:-1]] = i - 1
    val[rp[1:-1]] = -0.5
    col[rp[2:] - 1] = i
    val[rp[2:] - 1] = 2.0
    return rp, col, val


def _two_levels(n, top, dt, seed=9):
    """Rows >= top depend on 3 of the first `top` rows: level 1 holds n - top
    rows, more than the threads of the level solve's grid."""
    rng = np.random.default_rng(seed)
    lens = np.ones(n, np.int64)
    lens[top:] = 4
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    col = np.empty(rp[-1], np.int32)
    col[rp[:top]] = np.arange(top)
    offs = np.sort(rng.choice(top, size=(n - top, 3), replace=True), axis=1)
    col[rp[top]:] = np.concatenate([offs, np.arange(top, n)[:, None]], axis=1).ravel()
    val = rng.uniform(-0.3, 0.3, col.size).astype(dt)
    val[rp[1:] - 1] = 3.0
    return rp, col, val


@pytest.mark.parametrize("dt", [np.float32, np.float64])
@pytest.mark.parametrize("name", ["lap3d", "random_lower", "chain", "two_levels"])
def test_solves_bitexact(gpu, oracle, dt, name):
    if name == "lap3d":
        rp, col, val = synth.laplacian_3d_lower(24, dtype=dt)
    elif name == "chain":
        rp, col, val = _chain(20_000, dt)
    elif name == "two_levels":
        rp, col, val = _two_levels(300_000, 64, dt)
    else:
        rp, col, val = synth.random_lower(80_000, seed=3, band=2000, dtype=dt)
    N = rp.size - 1
    b = synth.uniform_vec(N, 4, dtype=dt)
    A = gpu.csr_from_host(rp, col, val)
    bv = gpu.vec_from_host(b)
    row_kernel = oracle.spts_csr(rp, col, val, b)
    syncfree = oracle.spts_syncfree(rp, col, val, b)
    truth = oracle.truth_spts(rp, col, val, b)
    for algo, want in (("level", row_kernel), ("hybrid", row_kernel), ("syncfree", syncfree)):
        yv = gpu.create_vec(N, 0, dt)
        gpu.spts(A, bv, yv, algo=algo)
        y = yv.array()
        assert np.array_equal(_ub(y), _ub(want)), algo
        rel = np.max(np.abs(y - truth)) / np.max(np.abs(truth))
        assert rel <= TOL[np.dtype(dt)] * 10, (algo, rel)


def test_f64_accumulation_policy(gpu, oracle):
    rp, col, val = synth.random_lower(50_000, seed=7, band=1000, dtype=np.float32)
    b = synth.uniform_vec(50_000, 1, dtype=np.float32)
    truth = oracle.truth_spts(rp, col, val, b)
    A = gpu.csr_from_host(rp, col, val)
    bv = gpu.vec_from_host(b)
    errs = {}
    for pol in ("native", "f64"):
        yv = gpu.create_vec(50_000, 0, np.float32)
        gpu.spts(A, bv, yv, algo="level", policy=pol)
        errs[pol] = np.max(np.abs(yv.array() - truth)) / np.max(np.abs(truth))
    assert errs["f64"] <= 1e-6 and errs["f64"] <= errs["native"]


def test_unsolvable_rejected(gpu):
    # diagonal not stored last in row 1
    A = gpu.csr_from_host([0, 1, 3], [0, 1, 0], np.array([1.0, 2.0, 3.0]))
    with pytest.raises(SparseError):
        gpu.spts(A, gpu.create_vec(2, 1.0, np.float64), gpu.create_vec(2, 0, np.float64))


def test_dependency_wait_times_out_and_device_stays_usable(gpu, oracle):
    """Row 2 lists itself before its diagonal: its ready flag can never be set
    before it is solved, so the bounded wait runs out; the call returns
    SB_ETIMEOUT and the next solve on the same device succeeds."""
    rp = np.array([0, 1, 3, 6], np.int32)
    col = np.array([0, 0, 1, 0, 2, 2], np.int32)
    val = np.array([2.0, 1.0, 4.0, 1.0, 1.0, 8.0])
    A = gpu.csr_from_host(rp, col, val)
    bv, yv = gpu.create_vec(3, 1.0, np.float64), gpu.create_vec(3, 0, np.float64)
    with pytest.raises(SparseError) as ei:
        gpu.spts_csr_sync_free(A, bv, yv, spin_limit_cycles=1 << 20)
    assert ei.value.status == -4
    good_rp, good_col, good_val = synth.laplacian_3d_lower(8)
    G = gpu.csr_from_host(good_rp, good_col, good_val)
    b = synth.uniform_vec(512, 2)
    yv = gpu.create_vec(512, 0, np.float64)
    gpu.spts_csr_sync_free(G, gpu.vec_from_host(b), yv)
    assert np.array_equal(_ub(yv.array()), _ub(oracle.spts_syncfree(good_rp, good_col,
                                                                     good_val, b)))
