"""Build libsparse_b200.so (all CUDA sources, sm_100a) in place.

    python -m sciwasm.sparse_b200.build

The library is a plain C-ABI shared object linked against the static CUDA
runtime; it carries no torch symbols.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
LIB = os.path.join(HERE, "libsparse_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libsparse_b200.so")


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")) +
                  glob.glob(os.path.join(HERE, "csrc", "*.cpp")))


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    """Compile every source to an object (in parallel, one nvcc per source)
    and link them into libsparse_b200.so; a no-op when the library is newer
    than every source and header."""
    srcs = sources()
    deps = srcs + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = ["-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC",
             "-Xcompiler", "-pthread", "-I", os.path.join(ROOT, "include"), *(extra or [])]
    objs = [os.path.join(objdir, os.path.basename(s) + ".o") for s in srcs]

    def compile_one(pair):
        src, obj = pair
        cmd = [nvcc_path(), *flags, "-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd), flush=True)
        return subprocess.run(cmd, capture_output=True, text=True)

    jobs = max(1, min(len(srcs), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=jobs) as pool:
        results = list(pool.map(compile_one, zip(srcs, objs)))
    for src, res in zip(srcs, results):
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise subprocess.CalledProcessError(res.returncode, f"nvcc {src}")
        if verbose and (res.stdout or res.stderr):
            sys.stderr.write(res.stdout + res.stderr)
    tmp = LIB + ".tmp"
    cmd = [nvcc_path(), *ARCH, "-Xcompiler", "-pthread", "-shared", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
