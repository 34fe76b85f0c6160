"""Build recipe for libkuqcd_b200.so (sm_100a) — compiles every CUDA source of the package in-tree.

    python -m kuqcd_b200.build          # or kuqcd_b200.build.build()

Each ``csrc/*.cu`` is compiled with ``nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` into
``_build/`` and linked into ``kuqcd_b200/libkuqcd_b200.so`` next to this file.  Objects are rebuilt only when a
source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libkuqcd_b200.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-ccbin", "/usr/bin/g++", f"-I{ROOT / 'include'}", f"-I{CSRC}", "--expt-relaxed-constexpr"]


def _headers():
    return list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((ROOT / "include").glob("*.h"))


def _stale(obj: Path, src: Path, hdr_mtime: float) -> bool:
    return not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_mtime)


def _compile(src: Path, extra: list[str]) -> Path:
    obj = BUILD / (src.stem + ".o")
    cmd = [NVCC, *ARCH, *FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)
    return obj


def build(verbose: bool = False, ptxas_info: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = sorted(CSRC.glob("*.cu"))
    hdr = max((h.stat().st_mtime for h in _headers()), default=0.0)
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    todo = [s for s in srcs if ptxas_info or _stale(BUILD / (s.stem + ".o"), s, hdr)]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            for obj in ex.map(lambda s: _compile(s, extra), todo):
                if verbose:
                    print("compiled", obj.name)
    objs = [BUILD / (s.stem + ".o") for s in srcs]
    if todo or not LIB.exists():
        cmd = [NVCC, *ARCH, "-shared", "-ccbin", "/usr/bin/g++", "-o", str(LIB), *map(str, objs),
               "-lcudart", "-Xlinker", "-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, ptxas_info="-v" in sys.argv))
