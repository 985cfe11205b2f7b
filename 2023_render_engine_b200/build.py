"""Builds the CUDA/C++ core into 2023_render_engine_b200/lib/librt_b200.so.

nvcc compiles every source in csrc/ for sm_100a (host code without FMA contraction,
so the host-side reference-order tree rounds like the reference's IEEE build), then
links one shared library exposing the C ABI of include/rt_b200.h.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT_DIR = HERE / "lib"
OBJ_DIR = HERE / "lib" / "obj"
LIB = OUT_DIR / "librt_b200.so"
INCLUDE = HERE.parent / "include"

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
          "--expt-relaxed-constexpr", "-I", str(INCLUDE)]


def _sources():
    return sorted([p for p in CSRC.iterdir() if p.suffix in (".cu", ".cpp")])


def _headers():
    return sorted([p for p in CSRC.iterdir() if p.suffix in (".h", ".cuh")]) + sorted(INCLUDE.glob("*.h"))


def _needs(obj: Path, src: Path, headers) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or any(h.stat().st_mtime > t for h in headers)


def _compile(src: Path, verbose_ptxas: bool) -> Path:
    obj = OBJ_DIR / (src.name + ".o")
    cmd = [NVCC, *COMMON, *ARCH, "-c", str(src), "-o", str(obj)]
    if src.suffix == ".cu":
        cmd += ["--extended-lambda"]
        if verbose_ptxas:
            cmd += ["-Xptxas", "-v"]
    else:
        cmd += ["-x", "cu"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> Path:
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    srcs = _sources()
    headers = _headers()
    todo = [s for s in srcs if force or _needs(OBJ_DIR / (s.name + ".o"), s, headers)]
    if todo:
        with cf.ThreadPoolExecutor(max_workers=min(8, len(todo))) as ex:
            list(ex.map(lambda s: _compile(s, verbose_ptxas), todo))
    objs = [OBJ_DIR / (s.name + ".o") for s in srcs]
    if todo or not LIB.exists():
        cmd = [NVCC, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose_ptxas="-v" in sys.argv))
