"""In-tree build of the CUDA library ``libbes.so`` for sm_100a.

Each kernel layout class (1, 2 or 4 units per lane on one warp; one unit
per lane on 2 or 4 warps) with each BiCG recurrence is its own translation
unit, so the objects compile in parallel; the shared library lands next to this
file so it travels with the source tree.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libbes.so"

KERNEL_UNITS = [f"bes_kernel_{c}{r}.cu" for c in ("u1", "u2", "u4", "g2", "g4") for r in ("", "_r1")]
SOURCES = ["bes_api.cu", "bes_launch.cu", "bes_peak.cu", "bes_noalloc.cu", "bes_mlp.cu", *KERNEL_UNITS]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    # every fused multiply-add in the solver is explicit; no contraction
    "--fmad=false",
    "-Xcompiler", "-fPIC",
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libbes.so")
    return cand


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [INCLUDE / "bes.h"]


def needs_build(lib: Path = LIB) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _deps())


def _compile(src: str, extra: list[str], outdir: Path) -> Path:
    obj = outdir / (Path(src).stem + ".o")
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", str(CSRC), "-I", str(INCLUDE), "-c", str(CSRC / src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{res.stderr}")
    return obj


def build(force: bool = False, extra_flags: list[str] | None = None, lib: Path = LIB, verbose: bool = False) -> Path:
    """Compile the CUDA sources and link ``libbes.so`` (skipped when up to date)."""
    if not force and not needs_build(lib):
        return lib
    extra = list(extra_flags or [])
    outdir = BUILD / (lib.stem if lib != LIB else "default")
    outdir.mkdir(parents=True, exist_ok=True)
    workers = min(len(SOURCES), os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(max_workers=workers) as ex:
        objs = list(ex.map(lambda s: _compile(s, extra, outdir), SOURCES))
    tmp = lib.with_suffix(".so.tmp")
    cmd = [nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp), *map(str, objs),
           "-lcudart"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc link failed:\n{res.stderr}")
    os.replace(tmp, lib)
    if verbose:
        print(f"built {lib}")
    return lib


if __name__ == "__main__":
    build(force=True, verbose=True)
