"""Builds the aero_b200 CUDA library (libaero_b200.so) in-tree with nvcc.

Every translation unit is compiled for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) with line info, in parallel,
into ``aero_b200/_build/``; the shared library is linked next to this file so
that it travels with the source tree.
"""

from __future__ import annotations

import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess

PKG = pathlib.Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
OUT_DIR = PKG / "_build"
LIB = PKG / "libaero_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
              "-Xcompiler", "-fvisibility=hidden"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found; the aero_b200 CUDA library cannot be built")
    return cand


def sources() -> list[pathlib.Path]:
    return sorted(list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cpp")))


def _headers() -> list[pathlib.Path]:
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h")))


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in sources() + _headers())


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> pathlib.Path:
    if not force and up_to_date():
        return LIB
    nvcc = _nvcc()
    OUT_DIR.mkdir(exist_ok=True)
    hdr_t = max(p.stat().st_mtime for p in _headers())

    def compile_one(src: pathlib.Path) -> pathlib.Path:
        obj = OUT_DIR / (src.name + ".o")
        if not force and obj.exists() and obj.stat().st_mtime >= max(src.stat().st_mtime, hdr_t):
            return obj
        extra = os.environ.get("AERO_NVCC_DEFINES", "").split()
        cmd = [nvcc, *NVCC_FLAGS, *extra, *ARCH, "-I", str(INCLUDE), "-c", str(src), "-o", str(obj)]
        if src.suffix == ".cpp":
            cmd = [nvcc, "-x", "cu", *cmd[1:]]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
        if verbose and (r.stderr.strip() or r.stdout.strip()):
            print(r.stdout, r.stderr)
        return obj

    jobs = jobs or min(8, os.cpu_count() or 4)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(compile_one, sources()))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-cudart", "static"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    import sys
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
