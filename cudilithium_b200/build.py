"""Builds the in-tree CUDA library ``cudilithium_b200/libcudilithium_b200.so`` for sm_100a.

Each ``csrc/*.cu`` translation unit (one per Dilithium parameter set plus the C-ABI unit) is
compiled in parallel with nvcc and linked into one shared library that exports the C ABI
declared in ``include/cudilithium.h``.  Run ``python cudilithium_b200/build.py`` (by path: importing
the package would load the library being built).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
ROOT = PKG.parent
LIB = PKG / "libcudilithium_b200.so"
OBJ_DIR = PKG / "_build"
LIB_BC = PKG / "libcudilithium_b200_bc.so"
OBJ_DIR_BC = PKG / "_build_bc"

NVCC_FLAGS = [
    "-O3",
    "-std=c++17",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo",
    "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC",
    "-I", str(ROOT / "include"),
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    deps = [src] + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "cudilithium.h"]
    t = obj.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps if d.exists())


def build(verbose: bool = False, force: bool = False, bounds_check: bool = False) -> Path:
    """Compiles and links the library; bounds_check=True makes the bounds-checked variant
    libcudilithium_b200_bc.so (device-side range checks, -DCUDIL_BOUNDS_CHECK) beside it."""
    nvcc = _nvcc()
    obj_dir = OBJ_DIR_BC if bounds_check else OBJ_DIR
    lib = LIB_BC if bounds_check else LIB
    flags = NVCC_FLAGS + (["-DCUDIL_BOUNDS_CHECK"] if bounds_check else [])
    obj_dir.mkdir(exist_ok=True)
    srcs = sources()
    jobs = []
    for s in srcs:
        o = obj_dir / (s.stem + ".o")
        if force or _stale(o, s):
            jobs.append((s, o))

    def run(job):
        s, o = job
        cmd = [nvcc, *flags, "-c", str(s), "-o", str(o)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {s.name}:\n{r.stdout}\n{r.stderr}")
        return o

    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 4))) as ex:
        list(ex.map(run, jobs))
    objs = [obj_dir / (s.stem + ".o") for s in srcs]
    if force or jobs or not lib.exists():
        cmd = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(lib), *map(str, objs),
               "-cudart", "static"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return lib


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv, bounds_check="--bounds-check" in sys.argv))
