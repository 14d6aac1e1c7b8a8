"""The C-ABI library loads and exports every symbol include/*.h declares;
without a GPU its entry points refuse loudly instead of computing on the CPU
(CPU only: no compute call is made)."""
import ctypes
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(sb_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_header_declares_functions():
    names = header_functions()
    assert "sb_spmv_csr" in names and "sb_malloc" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol(sb):
    from sciwasm.sparse_b200 import _lib
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (sb_\w+)", out))
    missing = [n for n in header_functions() if n not in exported]
    assert not missing, f"declared but not exported: {missing}"


def test_binding_covers_header(sb):
    from sciwasm.sparse_b200 import _lib
    assert set(header_functions()) <= set(_lib.declared_symbols())


def test_library_has_no_torch_dependency(sb):
    from sciwasm.sparse_b200 import _lib
    out = subprocess.run(["ldd", _lib.LIB_PATH], capture_output=True, text=True).stdout
    # library names and paths only: the load addresses in parentheses are
    # random hex that can contain "c10" by chance
    libs = [line.split("(")[0] for line in out.splitlines()]
    assert not any("torch" in lib or "c10" in lib for lib in libs), libs


def test_status_strings(sb):
    lib = sb.load_library()
    assert lib.sb_status_string(0) == b"ok"
    assert lib.sb_status_string(-3).startswith(b"refused")
    assert lib.sb_version() >= 10000


def test_invalid_arguments_rejected_before_device(sb):
    lib = sb.load_library()
    dummy = ctypes.c_void_p(16)
    assert lib.sb_spmv_csr(7, dummy, dummy, dummy, dummy, dummy, 4, 4, 1, None) == -1
    assert lib.sb_spmv_csr(0, dummy, dummy, dummy, dummy, dummy, -1, 4, 1, None) == -1
    assert b"dtype" in lib.sb_last_error() or b"negative" in lib.sb_last_error()


def test_no_cpu_fallback_without_device(sb):
    lib = sb.load_library()
    n = ctypes.c_int(-1)
    assert lib.sb_device_count(ctypes.byref(n)) == 0
    if n.value > 0:
        pytest.skip("a CUDA device is visible; this test covers the no-device path")
    dummy = ctypes.c_void_p(16)
    st = lib.sb_spmv_csr(0, dummy, dummy, dummy, dummy, dummy, 4, 4, 1, None)
    assert st == -6, lib.sb_last_error()
    p = ctypes.c_void_p()
    assert lib.sb_malloc(ctypes.byref(p), 64) == -6


def test_admission_predicates_match_oracle(sb, oracle):
    """sb_ell_admitted / sb_dia_admitted are host-only: same answers as the
    oracle's restatement of the reference's test on the known-answer cases."""
    import json
    k = json.load(open(os.path.join(ROOT, "tests", "golden", "kat_reference_semantics.json")))
    lib = sb.load_library()
    for c in k["admission"]["cases"]:
        if c["N"] > 2**31 - 1:
            continue
        assert bool(lib.sb_ell_admitted(c["w"], c["N"], c["nnz"])) == c["admitted"], c
        assert bool(lib.sb_dia_admitted(c["w"], c["N"], c["nnz"])) == c["admitted"], c
        assert oracle.format_admitted(c["w"], c["N"], c["nnz"]) == c["admitted"]
