"""Builds the library of the package: the CUDA kernels for sm_100a and the C++ host engine, into
o_o_solver_b200/_lib/liboosgpu.so (the C ABI of include/oos_gpu.h).

    python -m o_o_solver_b200.build            # build if any source is newer than the library
    python -m o_o_solver_b200.build --force
"""

from __future__ import annotations

import argparse
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PACKAGE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PACKAGE)
CSRC = os.path.join(PACKAGE, "csrc")
OUT_DIR = os.path.join(PACKAGE, "_lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIBRARY = os.path.join(OUT_DIR, "liboosgpu.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++20", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp,-O3", "-I" + os.path.join(ROOT, "include")]


def sources():
    found = []
    for folder in ("device", "host"):
        for name in sorted(os.listdir(os.path.join(CSRC, folder))):
            if name.endswith((".cu", ".cpp")):
                found.append(os.path.join(CSRC, folder, name))
    return found


def headers():
    found = [os.path.join(ROOT, "include", name) for name in os.listdir(os.path.join(ROOT, "include"))]
    for folder in ("device", "host"):
        for name in os.listdir(os.path.join(CSRC, folder)):
            if name.endswith((".cuh", ".hpp", ".h")):
                found.append(os.path.join(CSRC, folder, name))
    return found


def _object(source):
    rel = os.path.relpath(source, CSRC).replace(os.sep, "_")
    return os.path.join(OBJ_DIR, os.path.splitext(rel)[0] + ".o")


def _compile(source, verbose_ptxas=False):
    obj = _object(source)
    cmd = [NVCC, *ARCH, *COMMON, "-c", source, "-o", obj]
    if source.endswith(".cpp"):
        cmd = [NVCC, *COMMON, "-x", "cu", *ARCH, "-c", source, "-o", obj]
    if verbose_ptxas and source.endswith(".cu"):
        cmd.insert(1, "-Xptxas=-v")
    result = subprocess.run(cmd, capture_output=True, text=True)
    return source, result.returncode, result.stdout + result.stderr


def needs_build():
    if not os.path.exists(LIBRARY):
        return True
    built = os.path.getmtime(LIBRARY)
    return any(os.path.getmtime(path) > built for path in sources() + headers())


def build(force=False, verbose_ptxas=False, quiet=False):
    """Compiles every source for sm_100a and links the shared library; returns its path."""
    if not force and not needs_build():
        return LIBRARY
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = sources()
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        results = list(pool.map(lambda s: _compile(s, verbose_ptxas), srcs))
    failed = [r for r in results if r[1] != 0]
    for source, code, output in results:
        if output.strip() and (verbose_ptxas or code != 0) and not quiet:
            print(f"--- {os.path.relpath(source, ROOT)}\n{output}", file=sys.stderr)
    if failed:
        raise RuntimeError("nvcc failed: " + ", ".join(os.path.relpath(f[0], ROOT) for f in failed))
    link = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-o", LIBRARY, *[_object(s) for s in srcs]]
    result = subprocess.run(link, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError("link failed:\n" + result.stdout + result.stderr)
    return LIBRARY


def main():
    parser = argparse.ArgumentParser(description=__doc__)
    parser.add_argument("--force", action="store_true")
    parser.add_argument("--ptxas", action="store_true", help="print registers / spills / shared memory per kernel")
    args = parser.parse_args()
    print(build(force=args.force, verbose_ptxas=args.ptxas))


if __name__ == "__main__":
    main()
