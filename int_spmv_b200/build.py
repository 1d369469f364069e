"""Build recipe of libintspmv.so (in-tree, next to this file).

Host C (format builders, file I/O) is compiled with gcc -fopenmp; the CUDA
layer with nvcc for sm_100a only (`-gencode arch=compute_100a,code=sm_100a`),
then everything is linked into one shared library with a C ABI
(include/intspmv.h).  Rebuilds only when a source is newer than the library.

    python -m int_spmv_b200.build [--force]
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
LIB = PKG / "libintspmv.so"
OBJ = PKG / "_build"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-fvisibility=hidden,-fopenmp", "-Xptxas", "-warn-spills"]
CC_FLAGS = ["-O3", "-fPIC", "-fopenmp", "-fvisibility=hidden", "-std=gnu11", "-Wall", "-Wno-unknown-pragmas"]


def _cc() -> str:
    # The environment's $CC may lack OpenMP support files; the system gcc has them.
    return "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build int_spmv_b200")


# Sources compiled a second time with FPT = float (-DISPMV_FPT_FLOAT): the
# reference's API in its FP_TYPE=FP_FLOAT configuration, `_f32` symbols.
F32_SOURCES = ("builders.c", "io.c", "literal.cu", "harness.cu")


def sources() -> list[Path]:
    return sorted((CSRC / "host").glob("*.c")) + sorted((CSRC / "cuda").glob("*.cu"))


def units() -> list[tuple[Path, bool]]:
    """(source, FPT = float) for every object of the library."""
    return [(p, False) for p in sources()] + [(p, True) for p in sources() if p.name in F32_SOURCES]


def _deps() -> list[Path]:
    return sources() + sorted((CSRC / "cuda").glob("*.cuh")) + sorted(INCLUDE.glob("*.h"))


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _deps())


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build step failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def build(force: bool = False, verbose: bool = False) -> Path:
    if not force and not needs_build():
        return LIB
    OBJ.mkdir(exist_ok=True)
    nvcc, cc = _nvcc(), _cc()
    objs = []
    for src, f32 in units():
        obj = OBJ / (src.stem + ("_f32" if f32 else "") + (".c.o" if src.suffix == ".c" else ".cu.o"))
        defs = ["-DISPMV_FPT_FLOAT"] if f32 else []
        if src.suffix == ".c":
            cmd = [cc, *CC_FLAGS, *defs, f"-I{INCLUDE}", "-c", str(src), "-o", str(obj)]
        else:
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, *defs, f"-I{INCLUDE}", f"-I{CSRC / 'cuda'}", "-c", str(src), "-o",
                   str(obj)]
        if verbose:
            print(" ".join(cmd))
        _run(cmd)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-Xcompiler", "-fopenmp", "-o", str(tmp), *objs, "-lgomp", "-lm"]
    if verbose:
        print(" ".join(cmd))
    _run(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
