"""Reduced-precision storage: BF16 and f32 values with f32 accumulation.
Conversion is round-to-nearest-even (checked bit-exactly against a numpy
restatement); SpMV error is reported against FP64 of the stored (quantised)
values and of the original values.  <= 1e-5 is claimed only where it holds:
against the stored values, and for BF16-exact stencils against the originals."""
import numpy as np
import pytest

from conftest import rel_err
from sciwasm.sparse_b200 import synth

pytestmark = pytest.mark.gpu


def bf16_bits(a32):
    """Round f32 to bf16 (nearest, ties to even) -> uint16 words."""
    b = np.ascontiguousarray(a32, np.float32).view(np.uint32).astype(np.uint64)
    rounded = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return rounded.astype(np.uint16)


def bf16_to_f32(w):
    return (w.astype(np.uint32) << 16).view(np.float32)


def test_convert_values_bf16_round_to_nearest_even(gpu):
    rng = np.random.default_rng(0)
    v = np.concatenate([rng.standard_normal(100_000).astype(np.float32),
                        np.array([1.0, 1.00390625, 1.01171875, -3.5, 0.0, -0.0, 65504.0,
                                  1e-30, 3.4e38], np.float32)])
    d = gpu.DeviceArray.from_host(v)
    w = gpu.convert_values(d, "bf16").to_host()
    assert np.array_equal(w, bf16_bits(v))
    back = gpu.convert_values(gpu.DeviceArray.from_host(w), "f32").to_host()
    assert np.array_equal(back.view(np.uint32), bf16_to_f32(w).view(np.uint32))


@pytest.mark.parametrize("name", ["random", "powerlaw"])
def test_bf16_spmv_error_against_stored_and_original(gpu, oracle, name):
    if name == "random":
        rp, col, val = synth.banded(200_000, half=5, seed=3, dtype=np.float64)
    else:
        rp, col, val = synth.power_law(100_000, seed=4, dtype=np.float64, cap=2000)
    N = rp.size - 1
    x = synth.uniform_vec(N, 1, dtype=np.float32)
    A64 = gpu.csr_from_host(rp, col, val)
    A = gpu.csr_with_storage(A64, "bf16")
    xv, yv = gpu.vec_from_host(x), gpu.create_vec(N, 0, np.float32)
    gpu.spmv(A, xv, yv)
    y = yv.array()
    stored = bf16_to_f32(bf16_bits(val.astype(np.float32))).astype(np.float64)
    e_acc = rel_err(y, oracle.truth_csr(rp, col, stored, x.astype(np.float64)))
    e_all = rel_err(y, oracle.truth_csr(rp, col, val, x.astype(np.float64)))
    assert e_acc <= 1e-5, e_acc            # accumulation error (f32 sums)
    assert 1e-5 < e_all <= 2 ** -7, e_all  # BF16 quantisation dominates


def test_bf16_exact_stencil_meets_1e5_against_original(gpu, oracle):
    rp, col, val = synth.laplacian_2d(512, dtype=np.float32)  # 4 and -1: exact in BF16
    N = rp.size - 1
    x = synth.uniform_vec(N, 2, dtype=np.float32)
    A = gpu.csr_with_storage(gpu.csr_from_host(rp, col, val), "bf16")
    xv, yv = gpu.vec_from_host(x), gpu.create_vec(N, 0, np.float32)
    gpu.spmv(A, xv, yv)
    assert rel_err(yv.array(), oracle.truth_csr(rp, col, val, x)) <= 1e-5


def test_f32_long_rows_compensated(gpu, oracle):
    """Rows of 20,000 terms: the long-row path's compensated f32 sums stay
    within 1e-6 of the truth."""
    N = 64
    lens = np.full(N, 20_000)
    rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    rng = np.random.default_rng(5)
    col = rng.integers(0, N, rp[-1]).astype(np.int32)
    val = rng.uniform(0.5, 1.5, rp[-1]).astype(np.float32)
    x = rng.uniform(0.5, 1.5, N).astype(np.float32)
    A = gpu.csr_from_host(rp, col, val)
    xv, yv = gpu.vec_from_host(x), gpu.create_vec(N, 0, np.float32)
    gpu.spmv(A, xv, yv)
    assert rel_err(yv.array(), oracle.truth_csr(rp, col, val, x)) <= 1e-6
