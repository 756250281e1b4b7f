"""Builds libse.so (the sm_100a kernels behind include/se.h) in-tree with nvcc.

Every ``csrc/*.cu`` is compiled to an object for ``sm_100a`` (no PTX for other targets:
this library targets B200 only) and linked into ``scalingelections_b200/libse.so`` with the
static CUDA runtime, so the library has no dependency beyond the driver. Objects go to
``scalingelections_b200/_build/``. Rebuilds only what changed (source or common header
newer than the object).
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
BUILD = PKG / "_build"
LIB = PKG / "libse.so"
INCLUDE = PKG.parent / "include"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
    "-I",
    str(INCLUDE),
]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA 12.9 toolkit is required to build libse.so")
    return cand


def _deps(src: Path) -> list[Path]:
    return [src, *CSRC.glob("*.cuh"), INCLUDE / "se.h"]


def _needs(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(d.exists() and d.stat().st_mtime > t for d in _deps(src))


def _compile(nvcc: str, src: Path, obj: Path, extra: list[str]) -> None:
    cmd = [nvcc, *ARCH_FLAGS, *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")


def build(verbose: bool = False, extra_flags: list[str] | None = None) -> Path:
    """Compile and link libse.so; returns its path."""
    nvcc = nvcc_path()
    BUILD.mkdir(exist_ok=True)
    extra = list(extra_flags or [])
    sources = sorted(CSRC.glob("*.cu"))
    objs = [BUILD / (s.stem + ".o") for s in sources]
    todo = [(s, o) for s, o in zip(sources, objs) if _needs(o, s)]
    if todo:
        workers = max(1, min(len(todo), os.cpu_count() or 1))
        with cf.ThreadPoolExecutor(workers) as ex:
            futs = [ex.submit(_compile, nvcc, s, o, extra) for s, o in todo]
            for f in futs:
                f.result()
            if verbose:
                print(f"compiled {len(todo)} source(s)", file=sys.stderr)
    if todo or not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc, *ARCH_FLAGS, "-shared", "-cudart", "static", "-o", str(tmp), *map(str, objs)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc link failed:\n{r.stdout}\n{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
