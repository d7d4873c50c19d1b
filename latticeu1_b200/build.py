"""Build the sm_100a shared library behind the C ABI (include/u1_b200.h).

`python latticeu1_b200/build.py` compiles latticeu1_b200/csrc/*.cu with nvcc
into latticeu1_b200/lib/libu1b200.so (in-tree, so it travels with the
repository snapshot); `--checked` also builds the checked test library
libu1b200_check.so (-DU1_BOUNDS_CHECK).  No JIT cache is used.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
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


def _deps() -> list[Path]:
    deps = sources() + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "u1_b200.h"]
    return deps + sorted((PKG / "shim").rglob("*.cpp")) + sorted((PKG / "shim").rglob("*.h"))


def _compile_lib(target: Path, objdir: Path, defines: list[str], verbose: bool) -> None:
    """Every CUDA source (compiled in parallel) linked into `target`."""
    objdir.mkdir(parents=True, exist_ok=True)
    # -fmad=false: no compiler-chosen multiply-add contraction, so the
    # one-site, two-site and fused-measurement update kernels round every
    # link update identically (FMAs are written out where wanted).
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-Xcompiler", "-fPIC",
                    "-I" + str(ROOT / "include"), "-I" + str(CSRC),
                    "--expt-relaxed-constexpr"] + defines
    cmds, objs = [], []
    for src in sources():
        obj = objdir / (src.stem + ".o")
        cmds.append([nvcc()] + flags + ["-c", str(src), "-o", str(obj)])
        objs.append(str(obj))

    def run(cmd: list[str]) -> None:
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)

    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(run, c) for c in cmds]:
            f.result()
    tmp = target.with_suffix(".so.tmp")
    run([nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", str(tmp)] + objs)
    os.replace(tmp, target)


def build(force: bool = False, verbose: bool = False, extra: list[str] | None = None) -> Path:
    """Compile every CUDA source into one shared library; returns its path."""
    LIBDIR.mkdir(exist_ok=True)
    if not force and not _stale(LIB, _deps()):
        return LIB
    _compile_lib(LIB, LIBDIR / "obj", list(extra or []), verbose)
    build_shim(verbose=verbose)
    return LIB


CHECK_LIB = LIBDIR / "libu1b200_check.so"


def build_checked(force: bool = False, verbose: bool = False) -> Path:
    """The checked build (-DU1_BOUNDS_CHECK): the same sources with bounds and
    race checks on every link access of the update kernels, loaded instead of
    libu1b200.so when U1_CHECKED=1 (test infrastructure)."""
    LIBDIR.mkdir(exist_ok=True)
    if not force and not _stale(CHECK_LIB, _deps()):
        return CHECK_LIB
    _compile_lib(CHECK_LIB, LIBDIR / "obj_check", ["-DU1_BOUNDS_CHECK"], verbose)
    return CHECK_LIB


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
    if "--checked" in sys.argv:
        print(build_checked(force=force, verbose=True))
