"""sciwasm.sparse_b200 -- SciWasm.Sparse's sparse hot path on NVIDIA B200 (sm_100a).

Public API mirrors the reference's JavaScript module (spmv, coo_csr, csr_dia,
csr_ell, transpose, eliminate_zeros, element-wise maps, level sets, SpTS);
every operation runs as a CUDA kernel in libsparse_b200.so through its C ABI.
"""
from ._lib import SparseError, RefusedError, load as load_library  # noqa: F401
from .sparse import *  # noqa: F401,F403
from .sparse import (DeviceArray, sparse_COO_t, sparse_CSR_t, sparse_DIA_t,  # noqa: F401
                     sparse_ELL_t, sparse_vec_t)
