"""Builds the C-ABI shared library libunround_capi.so for sm_100a, in-tree.

nvcc compiles the CUDA kernels and the host driver (csrc/*.cu) and g++ the host model,
settings and C interface (csrc/*.cpp), all into unround/_native/libunround_capi.so, where
unround.native loads it (unless UNROUND_LIBRARY names another). Objects
go to _build/. The library links the CUDA runtime statically, so that it loads wherever the
driver is, and needs no torch.

Run: python jpeg-unround_b200/build.py [--force]
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCES = HERE / "csrc"
BUILD = HERE / "_build"
INCLUDE = HERE.parent / "include"
OUTPUT = HERE / "unround" / "_native" / "libunround_capi.so"
NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++20", "-I", str(INCLUDE), "-I", str(SOURCES)]
CUDA_FLAGS = [*ARCH, "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-O3"]
HOST_FLAGS = [*ARCH, "-x", "c++", "-Xcompiler", "-fPIC,-ffp-contract=off,-Wall"]


def _stale(target: Path, sources: list[Path]) -> bool:
    if not target.exists():
        return True
    built = target.stat().st_mtime
    return any(source.stat().st_mtime > built for source in sources)


def _compile(source: Path, force: bool) -> Path:
    target = BUILD / (source.name + ".o")
    headers = [*SOURCES.glob("*.hpp"), *SOURCES.glob("*.cuh"), *INCLUDE.rglob("*.h")]
    if force or _stale(target, [source, *headers]):
        flags = CUDA_FLAGS if source.suffix == ".cu" else HOST_FLAGS
        command = [NVCC, *COMMON, *flags, "-c", str(source), "-o", str(target)]
        subprocess.run(command, check=True)
    return target


def build(force: bool = False) -> Path:
    """Compiles what changed and links the library; returns its path."""
    BUILD.mkdir(exist_ok=True)
    OUTPUT.parent.mkdir(parents=True, exist_ok=True)
    sources = sorted([*SOURCES.glob("*.cu"), *SOURCES.glob("*.cpp")])
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
        objects = list(pool.map(lambda source: _compile(source, force), sources))
    if force or _stale(OUTPUT, objects):
        command = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", str(OUTPUT), *map(str, objects), "-lpthread", "-lz"]
        subprocess.run(command, check=True)
    return OUTPUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
