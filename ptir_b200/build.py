"""Build recipe of ``libptir_b200.so`` (nvcc, sm_100a, in-tree).

``python -m ptir_b200.build`` compiles every CUDA source of ``ptir_b200/csrc`` into one shared
library next to this file. Only nvcc and the CUDA toolkit headers are needed; no GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_PATH = os.path.join(HERE, "libptir_b200.so")
SOURCES = ("api.cu", "accel.cu", "tracer.cu", "wavefront.cu", "stages.cu", "storage.cu", "optim.cu", "envtable.cu")
ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS_COMPILE = ["-O3", "-lineinfo", "--use_fast_math", "-std=c++17", "-Xcompiler", "-fPIC"]
OBJ_DIR = os.path.join(HERE, "_build")


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libptir_b200.so")
    return path


def needs_build() -> bool:
    if not os.path.exists(LIB_PATH):
        return True
    t = os.path.getmtime(LIB_PATH)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "ptir_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, obj: str, verbose: bool) -> subprocess.CompletedProcess:
    cmd = [nvcc(), *ARCH_FLAGS, *NVCC_FLAGS_COMPILE, "-c", src, "-o", obj]
    if verbose:
        cmd[1:1] = ["-Xptxas", "-v"]
    return subprocess.run(cmd, capture_output=True, text=True)


def build(verbose: bool = False, force: bool = False) -> str:
    """Compile every source to an object in ptir_b200/_build (in parallel), then link the library."""
    if not force and not needs_build():
        return LIB_PATH
    from concurrent.futures import ThreadPoolExecutor

    os.makedirs(OBJ_DIR, exist_ok=True)
    objs = [os.path.join(OBJ_DIR, os.path.splitext(src)[0] + ".o") for src in SOURCES]
    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as pool:
        results = list(pool.map(lambda so: _compile(os.path.join(CSRC, so[0]), so[1], verbose), zip(SOURCES, objs)))
    failed = [r for r in results if r.returncode != 0]
    for r in results:
        if verbose or r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
    if failed:
        raise RuntimeError(f"nvcc failed ({len(failed)} of {len(SOURCES)} sources)")
    tmp = LIB_PATH + ".tmp"
    res = subprocess.run([nvcc(), *ARCH_FLAGS, "-shared", "-o", tmp, *objs], capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError(f"nvcc link failed ({res.returncode})")
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force=True)
    print(LIB_PATH)
