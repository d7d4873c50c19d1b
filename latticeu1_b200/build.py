"""Build the sm_100a shared library behind the C ABI (include/u1_b200.h).

`python latticeu1_b200/build.py` compiles latticeu1_b200/csrc/*.cu with nvcc
into latticeu1_b200/lib/libu1b200.so (in-tree, so it travels with the
repository snapshot).  No JIT cache is used.
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
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libu1b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libu1b200.so")
    return cand


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compile every CUDA source into one shared library; returns its path."""
    LIBDIR.mkdir(exist_ok=True)
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "u1_b200.h"]
    deps += sorted((PKG / "shim").rglob("*.cpp")) + sorted((PKG / "shim").rglob("*.h"))
    if not force and not _stale(LIB, deps):
        return LIB
    objdir = LIBDIR / "obj"
    objdir.mkdir(exist_ok=True)
    # -fmad=false: no compiler-chosen multiply-add contraction, so the
    # one-site, two-site and fused-measurement update kernels round every
    # link update identically (FMAs are written out where wanted).
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
                    "-I" + str(ROOT / "include"), "-I" + str(CSRC),
                    "--expt-relaxed-constexpr"] + (extra or [])
    objs = []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        cmd = [nvcc()] + flags + ["-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
        objs.append(str(obj))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", str(tmp)] + objs
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB)
    build_shim(verbose=verbose)
    return LIB


SHIM = PKG / "shim"
SHIM_LIB = LIBDIR / "libu1shim.so"


def build_shim(verbose: bool = False) -> Path:
    """The drop-in C++ API of the reference driver (namespace U1) over the
    C ABI: latticeu1_b200/lib/libu1shim.so, linked against libu1b200.so."""
    gxx = shutil.which("g++") if Path("/usr/bin/g++").exists() is False else "/usr/bin/g++"
    tmp = SHIM_LIB.with_suffix(".so.tmp")
    cmd = [gxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-I" + str(SHIM / "include"),
           "-I" + str(ROOT / "include")] + [str(p) for p in sorted(SHIM.glob("*.cpp"))] + [
           "-L" + str(LIBDIR), "-lu1b200", "-Wl,-rpath,$ORIGIN", "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, SHIM_LIB)
    return SHIM_LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose=True))
