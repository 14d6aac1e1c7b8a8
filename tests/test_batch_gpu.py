"""Batched SpMV: many uneven CSR matrices with 1..8 right-hand sides in one
graph-replayed persistent launch give the same results as one call per
matrix and right-hand side (within the stated tolerance)."""
import numpy as np
import pytest

from conftest import TOL, rel_err
from sciwasm.sparse_b200 import synth

pytestmark = pytest.mark.gpu


def _batch(seed, count, dt):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        N = int(np.exp(rng.uniform(np.log(500), np.log(20_000))))
        kind = i % 3
        if kind == 0:
            rp, col, val = synth.banded(N, half=int(rng.integers(1, 6)), seed=i, dtype=dt)
        elif kind == 1:
            rp, col, val = synth.power_law(N, seed=i, dtype=dt, cap=400, shift=2)
        else:
            rp, col, val = synth.laplacian_2d(int(np.sqrt(N)) + 1, dtype=dt)
        k = int(rng.integers(1, 9))
        out.append((rp, col, val, k))
    return out


@pytest.mark.parametrize("x_shift", ["none", "16B", "value"])
@pytest.mark.parametrize("storage,dt", [("f32", np.float32), ("f64", np.float64),
                                        ("bf16", np.float32)])
@pytest.mark.parametrize("lanes", [0, 1, 4])
def test_batch_matches_per_matrix(gpu, oracle, storage, dt, x_shift, lanes):
    """x 32-byte aligned: several right-hand sides load FP32 x rows in 32-byte
    blocks; 16 bytes off: 16-byte vectors or blocks; one value off (not
    16-byte aligned): nrhs lanes per row.  lanes 0 = the executor's choice,
    1 = one row per lane, 4 = four lanes interleaved over a row."""
    mats = _batch(7, 40, np.float64 if storage == "f64" else np.float32)
    ex = gpu.BatchExecutor(storage, capacity=64)
    jobs, host, keep = [], [], []
    for idx, (rp, col, val, k) in enumerate(mats):
        N = rp.size - 1
        A = gpu.csr_from_host(rp, col, val)
        if storage == "bf16":
            A = gpu.csr_with_storage(A, "bf16")
        vdt = np.float64 if storage == "f64" else np.float32
        X = synth.uniform_vec(N * k, idx, dtype=vdt).reshape(N, k)
        Y0 = synth.uniform_vec(N * k, 1000 + idx, dtype=vdt).reshape(N, k)
        if x_shift == "none":
            xd = gpu.DeviceArray.from_host(X.ravel())
            assert xd.ptr % 32 == 0
        else:
            pad = (16 if x_shift == "16B" else np.dtype(vdt).itemsize) // np.dtype(vdt).itemsize
            base = gpu.DeviceArray.from_host(np.concatenate([np.zeros(pad), X.ravel()]).astype(vdt))
            xd = gpu.DeviceArray(N * k, vdt, base.ptr + pad * np.dtype(vdt).itemsize)
            keep.append(base)  # the buffer must outlive the runs
        yd = gpu.DeviceArray.from_host(Y0.ravel())
        jobs.append((A, xd, yd, k))
        host.append((rp, col, val, X, Y0, A))
    for rep in range(2):  # graph replay: second run accumulates again
        ex.run(jobs, lanes=lanes)
        gpu.synchronize()
    tol = 1e-4 if storage == "bf16" else TOL[np.dtype(dt)]
    for (A, xd, yd, k), (rp, col, val, X, Y0, Ad) in zip(jobs, host):
        Y = yd.to_host().reshape(-1, k)
        vals = Ad.val_array()
        if storage == "bf16":
            vals = (vals.astype(np.uint32) << 16).view(np.float32)
        for j in range(k):
            once = oracle.truth_csr(rp, col, vals.astype(np.float64), X[:, j].astype(np.float64))
            want = Y0[:, j].astype(np.float64) + 2 * once
            assert rel_err(Y[:, j], want) <= tol * 4


def test_batch_same_result_alone_and_in_mix(gpu):
    """A matrix's result is the same when run alone and inside a batch."""
    mats = _batch(3, 12, np.float32)
    ex = gpu.BatchExecutor("f32", capacity=16)
    dev = []
    for i, (rp, col, val, k) in enumerate(mats):
        N = rp.size - 1
        X = synth.uniform_vec(N * k, i, dtype=np.float32)
        dev.append((gpu.csr_from_host(rp, col, val), gpu.DeviceArray.from_host(X), k, N))
    ys_mix = []
    jobs = []
    for A, xd, k, N in dev:
        yd = gpu.DeviceArray(N * k, np.float32)
        yd.fill_zero()
        jobs.append((A, xd, yd, k))
        ys_mix.append(yd)
    ex.run(jobs)
    gpu.synchronize()
    for (A, xd, k, N), ymix in zip(dev, ys_mix):
        yd = gpu.DeviceArray(N * k, np.float32)
        yd.fill_zero()
        ex.run([(A, xd, yd, k)])
        gpu.synchronize()
        assert np.array_equal(yd.to_host(), ymix.to_host())


def test_batch_back_to_back_runs(gpu):
    """The executor alternates two descriptor sets: four runs of different
    batches launched without a synchronisation in between (the third reuses
    the first one's set) each give the bits of the same batch run alone."""
    ex = gpu.BatchExecutor("f32", capacity=16)
    runs = []
    for r in range(4):
        jobs = []
        for i, (rp, col, val, k) in enumerate(_batch(20 + r, 6, np.float32)):
            N = rp.size - 1
            A = gpu.csr_from_host(rp, col, val)
            xd = gpu.DeviceArray.from_host(synth.uniform_vec(N * k, 50 * r + i, dtype=np.float32))
            yd = gpu.DeviceArray(N * k, np.float32)
            yd.fill_zero()
            jobs.append((A, xd, yd, k))
        runs.append(jobs)
    for jobs in runs:
        ex.run(jobs, overwrite=True)
    gpu.synchronize()
    together = [[yd.to_host() for _, _, yd, _ in jobs] for jobs in runs]
    for jobs, want in zip(runs, together):
        for A, xd, yd, k in jobs:
            yd.fill_zero()
        ex.run(jobs, overwrite=True)
        gpu.synchronize()
        for (A, xd, yd, k), w in zip(jobs, want):
            assert np.array_equal(yd.to_host(), w)


@pytest.mark.parametrize("storage", ["f32", "f64", "bf16"])
def test_batch_mixed_formats(gpu, oracle, storage):
    """CSR, DIA and ELL items in one launch.  With one right-hand side a DIA
    or ELL item is bit-identical to sb_spmv_dia / sb_spmv_ell on the same y;
    with several, each right-hand side is bit-identical to the oracle's serial
    DIA / ELL loop on that column; BF16 items are within tolerance of the FP64
    product of their stored values."""
    vdt = np.float64 if storage == "f64" else np.float32
    ex = gpu.BatchExecutor(storage, capacity=32)
    cases = []
    for i, (rp, col, val) in enumerate([synth.banded(7_001, half=3, seed=3, dtype=vdt),
                                        synth.laplacian_2d(90, dtype=vdt),
                                        synth.banded(40_000, half=5, seed=4, dtype=vdt)]):
        A = gpu.csr_from_host(rp, col, val)
        for fmt in ("dia", "ell", "csr"):
            M = {"dia": gpu.csr_dia, "ell": gpu.csr_ell, "csr": lambda a: a}[fmt](A)
            assert M is not None
            for k in (1, 3):
                cases.append((fmt, M, rp, col, val, k, i))
    jobs, host = [], []
    for idx, (fmt, M, rp, col, val, k, i) in enumerate(cases):
        N = rp.size - 1
        Ms = gpu.with_storage(M, "bf16") if storage == "bf16" else M
        X = synth.uniform_vec(N * k, 50 + idx, dtype=vdt).reshape(N, k)
        Y0 = synth.uniform_vec(N * k, 90 + idx, dtype=vdt).reshape(N, k)
        xd, yd = gpu.DeviceArray.from_host(X.ravel()), gpu.DeviceArray.from_host(Y0.ravel())
        jobs.append((Ms, xd, yd, k))
        host.append((fmt, M, Ms, rp, col, val, X, Y0))
    ex.run(jobs)
    gpu.synchronize()
    for (Ms, xd, yd, k), (fmt, M, _, rp, col, val, X, Y0) in zip(jobs, host):
        Y = yd.to_host().reshape(-1, k)
        N = M.N
        if storage == "bf16":
            v = (gpu.csr_with_storage(gpu.csr_from_host(rp, col, val), "bf16").val_array()
                 .astype(np.uint32) << 16).view(np.float32)
            for j in range(k):
                want = Y0[:, j].astype(np.float64) + oracle.truth_csr(
                    rp, col, v.astype(np.float64), X[:, j].astype(np.float64))
                assert rel_err(Y[:, j], want) <= 1e-4, (fmt, k)
            continue
        if fmt == "csr":
            for j in range(k):
                want = oracle.truth_csr(rp, col, val, X[:, j], Y0[:, j])
                assert rel_err(Y[:, j], want) <= TOL[np.dtype(vdt)], (fmt, k)
            continue
        for j in range(k):
            if fmt == "dia":
                want = oracle.spmv_dia(M.offset_array(), M.data_array(), N,
                                       np.ascontiguousarray(X[:, j]), Y0[:, j])
            else:
                want = oracle.spmv_ell(M.indices_array(), M.data_array(), N, M.ncols,
                                       np.ascontiguousarray(X[:, j]), Y0[:, j])
            assert np.array_equal(np.ascontiguousarray(Y[:, j]).view(np.uint8),
                                  want.view(np.uint8)), (fmt, k, j)
        if k == 1:
            xv, yv = gpu.vec_from_host(X[:, 0]), gpu.vec_from_host(Y0[:, 0])
            gpu.spmv(M, xv, yv)
            assert np.array_equal(yv.array().view(np.uint8),
                                  np.ascontiguousarray(Y[:, 0]).view(np.uint8)), fmt


@pytest.mark.parametrize("x_shift", ["none", "16B", "value"])
def test_gather_dot_rows_floor(gpu, x_shift):
    """sb_gather_dot_rows sums val[k] * (x row of col[k]) for 1..8 values per
    row with the batch kernel's loads (32-byte, 16-byte and unaligned x)."""
    import ctypes as C
    from sciwasm.sparse_b200 import _lib
    rng = np.random.default_rng(9)
    rows, nnz = 3001, 20_011
    col = rng.integers(0, rows, nnz).astype(np.int32)
    col[-1] = rows - 1  # the last x row, whose covering blocks would pass x's end
    val = rng.uniform(-1, 1, nnz).astype(np.float32)
    cd, vd = gpu.DeviceArray.from_host(col), gpu.DeviceArray.from_host(val)
    out = gpu.DeviceArray(1, np.float64)
    for K in range(1, 9):
        X = rng.uniform(-1, 1, rows * K).astype(np.float32)
        pad = {"none": 0, "16B": 4, "value": 1}[x_shift]
        base = gpu.DeviceArray.from_host(np.concatenate([np.zeros(pad, np.float32), X]))
        xptr = base.ptr + 4 * pad
        _lib.call("sb_gather_dot_rows", _lib.SB_F32, cd.ptr, vd.ptr, xptr, rows, K, nnz,
                  out.ptr, None)
        gpu.synchronize()
        got = float(out.to_host()[0])
        want = float(np.dot(val.astype(np.float64),
                            X.astype(np.float64).reshape(rows, K).sum(axis=1)[col]))
        assert abs(got - want) <= 1e-4 * max(1.0, np.sum(np.abs(val))), (K, got, want)
