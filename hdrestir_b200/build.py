"""Builds the sm_100a shared library ``libhdrestir_b200.so`` in-tree.

Every translation unit is compiled by nvcc with IEEE single/double arithmetic
in source order (-fmad=false, -prec-div/-prec-sqrt true, no flush-to-zero) and
host code with -ffp-contract=off: the kernels reproduce the reference's float
expressions operation by operation, so the compiler must not fuse or
reassociate them. Objects are rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "libhdrestir_b200.so"
INCLUDE = PKG.parent / "include"

SOURCES = ["hdr_abi.cpp", "host/scene_build.cpp", "host/shadow_bvh.cpp", "host/material_network.cpp", "raycast.cu", "integrate.cu", "wavefront.cu", "accumulate.cu",
           "accumulate_noalloc.cu", "server.cpp", "pathtrace.cu", "spatial.cu", "resolve.cu", "post.cu",
           "tlas.cu", "blas_build.cu", "wavefront_tex.cu"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-std=c++17", "-lineinfo",
    "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-I", str(INCLUDE),
]


def nvcc() -> str:
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build hdrestir_b200")
    return exe


def _headers() -> list[Path]:
    return list(CSRC.rglob("*.cuh")) + list(CSRC.rglob("*.h")) + list(INCLUDE.glob("*.h"))


def _stale(src: Path, obj: Path, newest_header: float) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or newest_header > t


def _compile(src: Path, obj: Path, verbose: bool) -> str:
    obj.parent.mkdir(parents=True, exist_ok=True)
    lang = ["-x", "cu"] if src.name == "hdr_abi.cpp" else []  # includes the device view types
    cmd = [nvcc(), *NVCC_FLAGS, *lang, "-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{res.stdout}\n{res.stderr}")
    return res.stderr


def build(verbose: bool = False, force: bool = False) -> Path:
    newest = max((h.stat().st_mtime for h in _headers()), default=0.0)
    jobs = []
    objs = []
    for rel in SOURCES:
        src = CSRC / rel
        obj = OBJ / (rel.replace("/", "_") + ".o")
        objs.append(obj)
        if force or _stale(src, obj, newest):
            jobs.append((src, obj))
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 4)) as ex:
            for (src, _), log in zip(jobs, ex.map(lambda j: _compile(j[0], j[1], verbose), jobs)):
                if verbose and log:
                    print(f"--- {src.name}\n{log}", file=sys.stderr)
    if jobs or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", str(LIB), *map(str, objs)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
