"""Build the sm_100a CUDA library in-tree: openturbine_b200/_lib/libkynema_b200.so.

    python -m openturbine_b200.build [--verbose]

nvcc cross-compiles for sm_100a without a GPU, so this runs on any host with
CUDA 12.9.  The library is self-contained (static cudart) and exports only the
C ABI of include/kynema_b200.h.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(OUT_DIR, "libkynema_b200.so")
SOURCES = ["kyn_capi.cu", "kyn_host.cpp"]
HEADERS = ["kyn_types.h", "kyn_host.hpp", "kyn_step_kernel.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA 12.9 toolkit is required to build")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "kynema_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps)


# Headers each source depends on (an object is rebuilt when one is newer).
DEPS = {
    "kyn_capi.cu": HEADERS,
    "kyn_host.cpp": ["kyn_types.h", "kyn_host.hpp"],
}


def _run(cmd: list[str], verbose: bool) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + res.stdout + res.stderr)
    if verbose:
        sys.stdout.write(res.stdout + res.stderr)


def build(verbose: bool = False, force: bool = False) -> str:
    """Compiles each source to an object (only those older than the source,
    its headers or include/kynema_b200.h, unless forced) and links the
    library."""
    if not force and not needs_build():
        return LIB
    obj_dir = os.path.join(OUT_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    base = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
            "-Xcompiler", "-fvisibility=hidden"]
    if os.path.exists("/usr/bin/g++"):
        base += ["-ccbin", "/usr/bin/g++"]
    api = os.path.join(HERE, "..", "include", "kynema_b200.h")
    objs = []
    for src in SOURCES:
        obj = os.path.join(obj_dir, src + ".o")
        deps = [os.path.join(CSRC, f) for f in [src] + DEPS[src]] + [api]
        stale = force or not os.path.exists(obj) or any(
            os.path.getmtime(d) > os.path.getmtime(obj) for d in deps)
        if stale:
            cmd = base + (["-Xptxas", "-v"] if verbose else []) + ["-c", os.path.join(CSRC, src), "-o", obj + ".tmp"]
            _run(cmd, verbose)
            os.replace(obj + ".tmp", obj)
        objs.append(obj)
    _run(base + ["-shared", "-o", LIB + ".tmp"] + objs, verbose)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
