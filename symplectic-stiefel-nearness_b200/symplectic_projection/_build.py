"""Build the native library ``libssn.so`` (sm_100a) from ``../csrc``.

Every ``.cu`` file under ``csrc`` is compiled with nvcc for
``arch=compute_100a,code=sm_100a`` and linked into one shared library placed
next to this file, so it ships with the package tree.  Objects go to
``csrc/_build`` (not version-controlled).  Cross-compiles without a GPU.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent                       # symplectic-stiefel-nearness_b200/
CSRC = ROOT / "csrc"
INCLUDE = ROOT.parent / "include"       # repository-level C ABI headers
OBJ = CSRC / "_build"
LIB = PKG / "libssn.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; set NVCC or add CUDA to PATH")


def _sources():
    return sorted(CSRC.glob("*.cu"))


def _deps():
    return list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))


def is_stale() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _deps())


def build(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile and link libssn.so if any source is newer than it."""
    if not force and not is_stale():
        return LIB
    nvcc = _nvcc()
    OBJ.mkdir(parents=True, exist_ok=True)
    flags = ARCH + FLAGS + [f"-I{INCLUDE}", f"-I{CSRC}"]

    def compile_one(src: Path) -> Path:
        obj = OBJ / (src.stem + ".o")
        cmd = [nvcc, *flags, "-c", str(src), "-o", str(obj)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stdout}\n{res.stderr}")
        if verbose:
            print(" ".join(cmd))
        return obj

    with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, _sources()))
    tmp = LIB.with_suffix(".so.tmp")
    # static CUDA runtime: the library does not depend on where libcudart lives
    cmd = [nvcc, *ARCH, "-shared", "--cudart", "static", "-o", str(tmp), *map(str, objs)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
