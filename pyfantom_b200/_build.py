"""Build the CUDA library in-tree: pyfantom_b200/libpyfantom_b200.so (sm_100a).

Each ``csrc/*.cu`` is compiled to an object with nvcc (parallel), then linked into one
shared library exporting the C ABI of ``include/pyfantom_b200.h``.  Objects go to
``pyfantom_b200/_build/``.  ``python -m pyfantom_b200._build [-v]`` rebuilds; ``-v`` also
prints the ptxas register / spill report.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libpyfantom_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
         "-I" + INCLUDE]


def _cutlass_include():
    """CuTe/CUTLASS headers vendored in the Python environment (used only to check the
    tensor-core descriptor encodings at run time); None if absent."""
    try:
        import importlib.util
        spec = importlib.util.find_spec("flashinfer")
        if spec and spec.origin:
            d = os.path.join(os.path.dirname(spec.origin), "data", "cutlass", "include")
            if os.path.exists(os.path.join(d, "cute", "arch", "mma_sm100_desc.hpp")):
                return d
    except Exception:
        pass
    return None


_CUTLASS = _cutlass_include()
if _CUTLASS:
    FLAGS.append("-I" + _CUTLASS)


def nvcc() -> str:
    cand = [os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), shutil.which("nvcc") or ""]
    for c in cand:
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found (set CUDA_HOME)")


def _sources():
    return sorted(glob.glob(os.path.join(SRC, "*.cu")))


def _headers():
    return sorted(glob.glob(os.path.join(SRC, "*.cuh"))) + [os.path.join(INCLUDE, "pyfantom_b200.h")]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _sources() + _headers() + [__file__])


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ, os.path.basename(src)[:-3] + ".o")
    cmd = [nvcc(), *ARCH, *FLAGS, "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stderr}")
    if verbose and r.stderr:
        print(r.stderr, file=sys.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), _sources()))
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose="-v" in sys.argv))
