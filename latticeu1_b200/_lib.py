"""ctypes binding of the C ABI declared in include/u1_b200.h.

The shared library is latticeu1_b200/lib/libu1b200.so, built in-tree by
latticeu1_b200/build.py.  With U1_CHECKED=1 in the environment the checked
build libu1b200_check.so (bounds and race checks on every link access of the
update kernels; a test build) is loaded instead.  There is no fallback: if
the library is missing or cannot be loaded, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

CHECKED = os.environ.get("U1_CHECKED", "0") not in ("", "0")
LIB_PATH = Path(__file__).resolve().parent / "lib" / ("libu1b200_check.so" if CHECKED else "libu1b200.so")

U1_OK = 0
U1_ERR_INVALID = -1
U1_ERR_CUDA = -2
U1_ERR_UNSUPPORTED = -3
U1_ERR_NOMEM = -4
U1_ERR_STATE = -5


class U1Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class u1_geom(C.Structure):
    _fields_ = [("dims", C.c_int), ("N", C.c_int * 4), ("beta", C.c_double), ("aniso", C.c_double)]


_vp = C.c_void_p
_i = C.c_int
_dp = C.POINTER(C.c_double)

# u1_dev_alloc_fn / u1_dev_free_fn (include/u1_b200.h)
DEV_ALLOC_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_size_t, C.POINTER(C.c_void_p))
DEV_FREE_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p)
NO_ALLOC, NO_FREE = DEV_ALLOC_FN(), DEV_FREE_FN()  # NULL function pointers

# name -> argtypes (all return int status unless listed in _RET)
SIGNATURES = {
    "u1_ctx_create": [_i, C.POINTER(_vp)],
    "u1_ctx_destroy": [_vp],
    "u1_ctx_set_stream": [_vp, _vp],
    "u1_geom_validate": [C.POINTER(u1_geom), C.POINTER(C.c_int64)],
    "u1_lattice_create": [_vp, C.POINTER(u1_geom), C.POINTER(_vp)],
    "u1_lattice_destroy": [_vp],
    "u1_lattice_set_stream": [_vp, _vp],
    "u1_lattice_info": [_vp, C.POINTER(C.c_int64)],
    "u1_lattice_set_coupling": [_vp, C.c_double, C.c_double],
    "u1_lattice_set_graphs": [_vp, _i],
    "u1_lattice_set_variant": [_vp, _i],
    "u1_lattice_get_variant": [_vp, C.POINTER(_i)],
    "u1_lattice_set_block": [_vp, _i],
    "u1_lattice_get_block": [_vp, C.POINTER(_i)],
    "u1_lattice_set_metropolis": [_vp, C.c_double, _i],
    "u1_lattice_get_metropolis": [_vp, _dp, C.POINTER(_i)],
    "u1_tune": [_vp, _vp, C.POINTER(_i)],
    "u1_lattice_links": [_vp, C.POINTER(_vp)],
    "u1_lattice_copy": [_vp, _vp],
    "u1_lattice_import_angles": [_vp, _vp, _i],
    "u1_lattice_export_angles": [_vp, _vp, _i],
    "u1_lattice_import_angles_async": [_vp, _vp, _i],
    "u1_lattice_export_angles_async": [_vp, _vp, _i],
    "u1_lattice_synchronize": [_vp],
    "u1_cold_start": [_vp],
    "u1_rng_create": [_vp, C.c_uint64, C.POINTER(_vp)],
    "u1_rng_destroy": [_vp],
    "u1_rng_get_state": [_vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)],
    "u1_rng_set_state": [_vp, C.c_uint64, C.c_uint64],
    "u1_rng_set_chain": [_vp, C.c_uint32],
    "u1_rng_set_replay": [_vp, _vp, C.c_size_t],
    "u1_rng_debug_uniforms": [_vp, _vp, C.c_uint64, _i, _i, _vp],
    "u1_hot_start": [_vp, _vp],
    "u1_update": [_vp, _vp, _i, _i],
    "u1_update_phase": [_vp, _vp, _i, _i, _i, _i],
    "u1_update_measure": [_vp, _vp, _i, _i, _vp],
    "u1_plaquette": [_vp, _dp],
    "u1_polyakov": [_vp, _dp],
    "u1_measure": [_vp, _dp],
    "u1_measure_async": [_vp, _vp],
    "u1_measure_noalloc": [_vp, C.POINTER(u1_geom), _vp, _vp],
    "u1_poly_corr": [_vp, _i, _dp, _i],
    "u1_multilevel": [_vp, _vp, _i, _i, _i, _i, _i, _i, _dp, _i],
    "u1_batch_create": [_vp, _i, C.POINTER(u1_geom), C.c_uint64, C.c_uint32, C.POINTER(_vp)],
    "u1_batch_destroy": [_vp],
    "u1_batch_set_stream": [_vp, _vp],
    "u1_batch_info": [_vp, C.POINTER(C.c_int64)],
    "u1_batch_groups": [_vp, C.POINTER(_i)],
    "u1_batch_tune": [_vp, C.POINTER(_i)],
    "u1_batch_configure": [_vp, _i, _i, C.POINTER(_i), C.POINTER(_i)],
    "u1_batch_group_info": [_vp, _i, C.POINTER(_i)],
    "u1_batch_set_lanes": [_vp, _i],
    "u1_batch_get_lanes": [_vp, C.POINTER(_i)],
    "u1_batch_hot_start": [_vp],
    "u1_batch_update": [_vp, _i, _i, _i],
    "u1_batch_measure": [_vp, _dp],
    "u1_batch_results": [_vp, _dp],
    "u1_batch_results_device": [_vp, C.POINTER(_vp)],
    "u1_batch_import_angles": [_vp, _i, _vp],
    "u1_batch_export_angles": [_vp, _i, _vp],
    "u1_batch_get_pass": [_vp, C.POINTER(C.c_uint64)],
    "u1_batch_export_all": [_vp, _vp],
    "u1_action_workspace_bytes": [C.POINTER(u1_geom), _i, C.POINTER(C.c_size_t)],
    "u1_wilson_action": [C.POINTER(u1_geom), _vp, _i, _i, _vp, _vp, _vp],
    "u1_wilson_action_grad": [C.POINTER(u1_geom), _vp, _i, _i, _vp, _vp, _vp],
    "u1_convert_order": [C.POINTER(u1_geom), _vp, _vp, _i, _vp],
    "u1_plaquette_fields": [_vp, _i, _vp, _dp],
    "u1_checkpoint_save": [_vp, _vp, C.c_char_p, _i],
    "u1_checkpoint_load": [_vp, _vp, C.c_char_p],
    "u1_checkpoint_info": [C.c_char_p, C.POINTER(u1_geom), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                           C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)],
    "u1_ncp_forward": [_vp, _vp, C.c_int64, _i, _vp, _vp, _vp],
    "u1_ncp_backward": [_vp, _vp, _vp, _vp, C.c_int64, _i, _vp, _vp, _vp],
    "u1_ncp_inverse": [_vp, _vp, C.c_int64, _i, _vp, _vp, _vp, _vp],
    "u1_ncp_inverse_backward": [_vp, _vp, _vp, _vp, C.c_int64, _i, _vp, _vp, _vp],
    "u1_flow_layer_forward": [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, C.c_float, _vp],
    "u1_flow_layer_inverse": [_vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, C.c_float, _vp],
    "u1_flow_layer_inverse_backward": [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp,
                                       C.c_float, _vp],
    "u1_flow_layer_backward": [_vp, _vp, _vp, _vp, _vp, _vp, _i, _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, C.c_float,
                               _vp],
    "u1_kernel_launch_count": [C.POINTER(C.c_uint64)],
    "u1_set_device_allocator": [DEV_ALLOC_FN, DEV_FREE_FN, _vp],
    "u1_device_allocations": [C.POINTER(C.c_int64)],
    "u1_lattice_set_wave_wait": [_vp, C.c_uint, _i],
    "u1_check_report": [_vp, C.POINTER(C.c_int64), _i],
    "u1_check_selftest": [_vp, C.POINTER(C.c_int64)],
    "u1_last_error": [],
    "u1_version": [],
}
_RET = {"u1_last_error": C.c_char_p, "u1_version": C.c_char_p}


def load(path: Path = LIB_PATH) -> C.CDLL:
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build it with `python latticeu1_b200/build.py` "
            "(the CUDA path has no CPU fallback)")
    lib = C.CDLL(str(path))
    for name, argtypes in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = _RET.get(name, C.c_int)
    return lib


lib = load()


def last_error() -> str:
    return (lib.u1_last_error() or b"").decode()


def check(rc: int, what: str = "") -> None:
    if rc != U1_OK:
        raise U1Error(rc, f"{what}: {last_error()}" if what else last_error())


def device_allocations() -> int:
    """Device blocks the library currently holds."""
    v = C.c_int64(0)
    check(lib.u1_device_allocations(C.byref(v)), "u1_device_allocations")
    return int(v.value)


def launch_count() -> int:
    v = C.c_uint64(0)
    check(lib.u1_kernel_launch_count(C.byref(v)), "u1_kernel_launch_count")
    return int(v.value)


def check_report(ctx, reset: bool = False) -> dict:
    """Counters of the checked build (U1_CHECKED=1): bounds violations,
    races, phases checked, links accessed and the first violation."""
    out = (C.c_int64 * 8)()
    check(lib.u1_check_report(ctx, out, 1 if reset else 0), "u1_check_report")
    return _check_dict(out)


def check_selftest(ctx) -> dict:
    """The checked build's checks on a planted 16-link case (u1_check_selftest)."""
    out = (C.c_int64 * 8)()
    check(lib.u1_check_selftest(ctx, out), "u1_check_selftest")
    return _check_dict(out)


def _check_dict(out) -> dict:
    keys = ("bad", "races", "phases", "marked", "first_bad_idx", "first_bad_half", "first_bad_kind",
            "first_race_link")
    return {k: int(v) for k, v in zip(keys, out)}
