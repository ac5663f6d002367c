"""Build step: compiles csrc/ into the in-tree shared library libspk_b200.so.

    python cpp-max-packer_b200/build.py [--force]

Every CUDA source is compiled for sm_100a only
(-gencode arch=compute_100a,code=sm_100a) with -lineinfo; host code keeps
IEEE binary64 semantics (-ffp-contract=off) because the rasteriser's interval
arithmetic must round exactly like the reference's.
"""

from __future__ import annotations

import concurrent.futures as futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libspk_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
          "-Xcompiler", "-ffp-contract=off", "-I", os.path.join(HERE, "..", "include")]


def sources():
    return sorted(f for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers_mtime():
    return max(os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC)
               if f.endswith((".cuh", ".hpp", ".h")))


def compile_one(name, force):
    src = os.path.join(CSRC, name)
    obj = os.path.join(OBJ, name + ".o")
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), headers_mtime()):
        return obj, None
    extra = ["-x", "cu"] if name.endswith(".cu") else ["-x", "c++"]
    cmd = [NVCC, *ARCH, *COMMON, *extra, "-c", src, "-o", obj]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode:
        return obj, f"{' '.join(cmd)}\n{proc.stdout}{proc.stderr}"
    return obj, None


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    names = sources()
    with futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        results = list(pool.map(lambda n: compile_one(n, force), names))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("CUDA build failed:\n" + "\n".join(errors))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        proc = subprocess.run(cmd, capture_output=True, text=True)
        if proc.returncode:
            raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{proc.stdout}{proc.stderr}")
    if verbose:
        print(LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
