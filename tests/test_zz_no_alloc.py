"""u1_measure_noalloc: the measurement for callers that cannot allocate.

Some callers cannot call cudaMalloc, for example code confined to memory its
host framework hands out, or loops that cannot accept a cudaMalloc that may
synchronise the device.  u1_measure_noalloc runs the same fused plaquette +
Polyakov kernel as u1_measure_async with its scratch in a fixed device array
inside the library (lattices up to V/2 = 1,048,576 sites).  Here it is called
through the C ABI and compared, on two calls in a row, with the existing
entry point; the file is collected last so a stop-at-first-failure run has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from latticeu1_b200 import _lib
from latticeu1_b200._lib import lib, u1_geom

TOL = 2e-6  # the measurement tolerance used by the other GPU tests


def _geom(dims, N, beta=1.0, aniso=1.0):
    return u1_geom(dims=dims, N=(C.c_int * 4)(*N), beta=beta, aniso=aniso)


def test_noalloc_rejects_lattice_above_limit_before_device_work():
    """V/2 above the fixed array's capacity is refused by the host-side check,
    which runs before any CUDA call (so this also runs without a GPU)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("checked here only where no GPU is present")
    g = _geom(4, (48, 48, 48, 48))
    dummy = C.c_void_p(256)
    rc = lib.u1_measure_noalloc(dummy, C.byref(g), dummy, None)
    assert rc == _lib.U1_ERR_INVALID
    assert "too large" in _lib.last_error()


@pytest.mark.gpu
def test_noalloc_matches_measure_on_two_calls():
    import torch

    from latticeu1_b200 import Context, Lattice, Rng

    ctx = Context(0)
    out = torch.zeros(6, dtype=torch.float64, device="cuda")
    cases = [(4, (16, 16, 16, 16), 1.0, 1.0), (3, (12, 8, 0, 10), 2.0, 1.3)]
    for call, (dims, N, beta, aniso) in enumerate(cases):
        lat = Lattice(ctx, dims, N, beta, aniso)
        rng = Rng(ctx, 100 + call)
        lat.hot_start(rng)
        lat.update(rng, 1, 4)
        want = lat.measure()          # existing entry point (library-owned scratch)
        torch.cuda.synchronize()
        out.fill_(np.nan)
        torch.cuda.synchronize()
        g = _geom(dims, list(N) + [0] * (4 - len(N)), beta, aniso)
        rc = lib.u1_measure_noalloc(C.c_void_p(lat.links_ptr()), C.byref(g), C.c_void_p(out.data_ptr()), None)
        assert rc == 0, _lib.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert abs(complex(got[0], got[1]) - want["plaq_ss"]) < TOL, (call, got, want)
        assert abs(complex(got[2], got[3]) - want["plaq_st"]) < TOL, (call, got, want)
        assert abs(complex(got[4], got[5]) - want["poly"]) < TOL, (call, got, want)
        lat.close()
        rng.close()
