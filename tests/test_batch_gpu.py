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


@pytest.mark.parametrize("storage,dt", [("f32", np.float32), ("f64", np.float64),
                                        ("bf16", np.float32)])
def test_batch_matches_per_matrix(gpu, oracle, storage, dt):
    mats = _batch(7, 40, np.float64 if storage == "f64" else np.float32)
    ex = gpu.BatchExecutor(storage, capacity=64)
    jobs, host = [], []
    for idx, (rp, col, val, k) in enumerate(mats):
        N = rp.size - 1
        A = gpu.csr_from_host(rp, col, val)
        if storage == "bf16":
            A = gpu.csr_with_storage(A, "bf16")
        vdt = np.float64 if storage == "f64" else np.float32
        X = synth.uniform_vec(N * k, idx, dtype=vdt).reshape(N, k)
        Y0 = synth.uniform_vec(N * k, 1000 + idx, dtype=vdt).reshape(N, k)
        xd, yd = gpu.DeviceArray.from_host(X.ravel()), gpu.DeviceArray.from_host(Y0.ravel())
        jobs.append((A, xd, yd, k))
        host.append((rp, col, val, X, Y0, A))
    for rep in range(2):  # graph replay: second run accumulates again
        ex.run(jobs)
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
