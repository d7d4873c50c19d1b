"""CPU-only checks of the C-ABI library: it loads, exports every symbol the
headers in include/ declare, validates geometry on the host, and fails
cleanly (status code + message, no crash) when no GPU is present."""
import ctypes as C
import re
from pathlib import Path

import pytest

import latticeu1_b200 as u1
from latticeu1_b200 import _lib

INCLUDE = Path(__file__).resolve().parents[1] / "include"


def declared_symbols():
    names = set()
    for h in INCLUDE.glob("*.h"):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s*(u1_\w+)\s*\(", text, flags=re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "u1_update" in names and "u1_multilevel" in names and len(names) > 25


@pytest.mark.parametrize("name", declared_symbols())
def test_library_exports_symbol(name):
    assert hasattr(_lib.lib, name), f"{name} declared in include/ but not exported"


def test_every_exported_entry_point_is_declared_and_bound():
    """The reverse direction: every extern "C" u1_* definition in the sources
    is declared in include/ and has argtypes in the ctypes stub."""
    csrc = Path(__file__).resolve().parents[1] / "latticeu1_b200" / "csrc"
    defined = set()
    for f in list(csrc.glob("*.cu")) + list(csrc.glob("*.cpp")):
        defined |= set(re.findall(r'extern "C"\s+(?:const\s+)?\w+\s*\**\s*(u1_\w+)\s*\(', f.read_text()))
    assert len(defined) > 25
    declared = set(declared_symbols())
    assert not defined - declared, sorted(defined - declared)
    assert not defined - set(_lib.SIGNATURES) - set(getattr(_lib, "_RET", {})), \
        sorted(defined - set(_lib.SIGNATURES))


def _geom(dims, N, beta=1.0, aniso=1.0):
    return _lib.u1_geom(dims=dims, N=(C.c_int * 4)(*N), beta=beta, aniso=aniso)


@pytest.mark.parametrize("dims,N,expect", [
    (4, (32, 32, 32, 32), [32 ** 4, 32 ** 4 // 2, 32 ** 3, 4, 32, 32, 32, 32]),
    (4, (24, 24, 24, 48), [24 ** 3 * 48, 24 ** 3 * 24, 24 ** 3, 4, 24, 24, 24, 48]),
    (3, (6, 4, 99, 8), [192, 96, 24, 3, 6, 4, 8, 1]),
    (2, (32, 7, 7, 16), [512, 256, 32, 2, 32, 16, 1, 1]),
])
def test_geom_validate_matches_reference_grid(dims, N, expect):
    out = (C.c_int64 * 8)()
    assert _lib.lib.u1_geom_validate(C.byref(_geom(dims, N)), out) == 0
    assert list(out) == expect


@pytest.mark.parametrize("dims,N", [(4, (32, 31, 32, 32)), (2, (8, 0, 0, 5)), (5, (4, 4, 4, 4)), (1, (4, 4, 4, 4))])
def test_geom_validate_rejects(dims, N):
    out = (C.c_int64 * 8)()
    rc = _lib.lib.u1_geom_validate(C.byref(_geom(dims, N)), out)
    assert rc == _lib.U1_ERR_INVALID
    assert _lib.last_error()


def test_geom_validate_rejects_bad_aniso():
    assert _lib.lib.u1_geom_validate(C.byref(_geom(4, (4, 4, 4, 4), aniso=0.0)), None) == _lib.U1_ERR_INVALID


def test_version_and_launch_counter():
    assert b"sm_100a" in _lib.lib.u1_version()
    assert u1.launch_count() >= 0


def test_ctx_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    rc = _lib.lib.u1_ctx_create(0, C.byref(h))
    assert rc != 0 and not h.value
    assert _lib.last_error()
    with pytest.raises(u1.U1Error):
        u1.Context(0)


def test_null_arguments_return_invalid():
    assert _lib.lib.u1_update(None, None, 1, 4) == _lib.U1_ERR_INVALID
    assert _lib.lib.u1_measure(None, None) == _lib.U1_ERR_INVALID
    assert _lib.lib.u1_multilevel(None, None, 1, 1, 1, 1, 1, 1, None, 0) == _lib.U1_ERR_INVALID


def test_integration_example_compiles(tmp_path):
    """The C ABI example of INTEGRATION.md compiles against include/u1_b200.h
    (g++ -fsyntax-only; no device needed)."""
    import shutil
    import subprocess
    root = Path(__file__).resolve().parents[1]
    text = (root / "INTEGRATION.md").read_text()
    m = re.search(r"```c\+\+\n(.*?)```", text, re.S)
    assert m, "no C++ example in INTEGRATION.md"
    body = m.group(1).replace('#include "u1_b200.h"', "")
    src = tmp_path / "example.cpp"
    src.write_text('#include "u1_b200.h"\nint main() {\n' + body + "return 0;\n}\n")
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not found")
    r = subprocess.run([gxx, "-std=c++17", "-fsyntax-only", "-Wall", "-I" + str(root / "include"), str(src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
