"""TEST INFRASTRUCTURE: build recipe for the reference's own CUDA solver.

Compiles oracle/ref_harness.cu against the reference's unmodified headers in
place (the reference tree and its ``SourceCodes`` directory, given as an
argument or by the environment variable ``BES_REFERENCE_DIR``) with the
reference's own nvcc flags (makefile:2), except ``sm_100a`` for ``sm_35``.
Outputs go to ``oracle/_ref/`` only (git-ignored; the built binaries travel
with the tree to the GPU machine, the reference sources do not).

Variants: ``ref_n{UPS}_s{NS}_d{NDO}`` with the shipped ``-maxrregcount=128``
and ``..._nocap`` without it.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
MARKER = OUT / "reference_dir.txt"   # the tree the last build() used (git-ignored, like the binaries)


def reference_dir(given=None):
    """The reference tree: the argument, else $BES_REFERENCE_DIR, else the tree
    the last build() used, else None."""
    d = given or os.environ.get("BES_REFERENCE_DIR")
    if not d and MARKER.exists():
        d = MARKER.read_text().strip()
    return Path(d) if d else None

# (units per system, max systems, dense-output slots, register cap)
VARIANTS = [
    (32, 256, 0, True), (32, 256, 0, False),
    (32, 64, 16, True),
    (64, 64, 0, True),
    (128, 16, 0, True),
    (128, 4096, 0, True), (128, 4096, 0, False),   # configuration 3: 4096 systems sharing one matrix
]


def name(ups: int, ns: int, ndo: int, cap: bool) -> str:
    return f"ref_n{ups}_s{ns}_d{ndo}" + ("" if cap else "_nocap")


def path(ups: int, ns: int, ndo: int = 0, cap: bool = True) -> Path:
    return OUT / name(ups, ns, ndo, cap)


def available(reference=None) -> bool:
    ref = reference_dir(reference)
    return ref is not None and (ref / "SourceCodes" / "CoupledSystems_PerBlock_Interface.cuh").exists()


def _one(v, ref: Path) -> Path:
    ups, ns, ndo, cap = v
    exe = path(ups, ns, ndo, cap)
    src = HERE / "ref_harness.cu"
    if exe.exists() and exe.stat().st_mtime > src.stat().st_mtime:
        return exe
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-O3", "--std=c++11", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-w",
           f"-DHARNESS_UPS={ups}", f"-DHARNESS_NS={ns}", f"-DHARNESS_NDO={ndo}",
           "-I", str(ref), "-I", str(ref / "SourceCodes"), str(src), "-o", str(exe)]
    if cap:
        cmd.insert(1, "-maxrregcount=128")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"reference build failed ({exe.name}):\n{res.stderr[-4000:]}")
    return exe


DROPIN = [(32, 256, 0), (32, 64, 16)]


def dropin_path(ups: int, ns: int, ndo: int = 0) -> Path:
    return OUT / f"dropin_n{ups}_s{ns}_d{ndo}"


def build_dropin() -> list[Path]:
    """The same driver (ref_harness.cu) compiled against include/dropin/, i.e.
    the C++ ProblemSolver shim over libbes.so instead of the reference headers.
    Needs no reference tree."""
    OUT.mkdir(exist_ok=True)
    root = HERE.parent
    pkg = root / "bubbleensemble_implicitextension_b200"
    src = HERE / "ref_harness.cu"
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    outs = []
    for ups, ns, ndo in DROPIN:
        exe = dropin_path(ups, ns, ndo)
        deps = [src, root / "include" / "bes_problem_solver.h", root / "include" / "bes.h", pkg / "libbes.so"]
        if exe.exists() and all(exe.stat().st_mtime > d.stat().st_mtime for d in deps if d.exists()):
            outs.append(exe)
            continue
        cmd = [nvcc, "-O2", "--std=c++17", "-w", f"-DHARNESS_UPS={ups}", f"-DHARNESS_NS={ns}", f"-DHARNESS_NDO={ndo}",
               "-I", str(root / "include" / "dropin"), "-I", str(root / "include"), str(src), "-o", str(exe),
               "-L", str(pkg), "-lbes", "-Xlinker", "-rpath=$ORIGIN/../../bubbleensemble_implicitextension_b200"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"drop-in build failed ({exe.name}):\n{res.stderr[-4000:]}")
        outs.append(exe)
    return outs


def build(reference=None) -> list[Path]:
    """Build every variant from the reference tree `reference` (default
    $BES_REFERENCE_DIR); a no-op when no reference tree is given or found."""
    if not available(reference):
        return []
    ref = reference_dir(reference)
    OUT.mkdir(exist_ok=True)
    MARKER.write_text(str(ref) + "\n")
    with cf.ThreadPoolExecutor(max_workers=min(len(VARIANTS), os.cpu_count() or 1)) as ex:
        return list(ex.map(lambda v: _one(v, ref), VARIANTS))


# the reference's own drivers and the -D flags they need (BubbleEnsemble.cu uses NCOLL,
# which only CollapseStrength.cu defines)
DRIVERS = {"CollapseStrength": [], "BubbleEnsemble": ["-DNCOLL=32"]}


def build_reference_drivers(outdir: Path, reference=None) -> dict:
    """Compile the reference's own driver programs, unchanged, against
    include/dropin/ and link them with libbes.so (the drop-in: the drivers'
    ProblemSolver<...> runs on this library).  Returns {driver: executable};
    empty when no reference tree is found."""
    ref = reference_dir(reference)
    if ref is None or not (ref / "CollapseStrength.cu").exists():
        return {}
    root = HERE.parent
    pkg = root / "bubbleensemble_implicitextension_b200"
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    outdir.mkdir(parents=True, exist_ok=True)
    out = {}
    for drv, flags in DRIVERS.items():
        exe = outdir / f"dropin_{drv}"
        cmd = [nvcc, "-O2", "--std=c++17", "-w", *flags, "-I", str(root / "include" / "dropin"),
               "-I", str(root / "include"), str(ref / f"{drv}.cu"), "-o", str(exe),
               "-L", str(pkg), "-lbes", "-Xlinker", f"-rpath={pkg}"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"{drv}.cu does not build against the drop-in:\n{res.stderr[-4000:]}")
        out[drv] = exe
    return out


if __name__ == "__main__":
    import sys
    for p in build(sys.argv[1] if len(sys.argv) > 1 else None):
        print(p)
